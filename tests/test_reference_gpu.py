"""The reference's own GPU kernels (oracle/_ref/libref_gpu.so, built from
cuda_BackProjectionKernels.cuh by oracle/Makefile) as the timed reference-GPU
baseline: its guard against the kernel's index -1 read, and its image against
the FP64 path on the point-target configuration."""
import numpy as np
import pytest

from oracle import oracle as O
from uncc_sar_focusing_b200 import scenes as S

needs_lib = pytest.mark.skipif(not O.ref_gpu_available(), reason="oracle/_ref/libref_gpu.so not built")


@needs_lib
def test_guard_refuses_scene_at_swath_edge():
    # a 200 m wide image in a 105.7 m swath: pixels reach the lower edge, where
    # the reference kernel's roundf bracket would read index -1; refused on the
    # host before any device work
    sc = S.point_target_scene(K=64, Np=16, n=32, spacing=0.1, nfft=256, snr_db=None, seed=1, n_targets=1)
    sc.grid = S.Grid(nx=32, ny=32, wx=200.0, wy=200.0)
    with pytest.raises(ValueError, match="swath"):
        O.reference_gpu_focus(sc, reps=1)


@needs_lib
@pytest.mark.gpu
def test_reference_gpu_image_focuses_like_fp64():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from uncc_sar_focusing_b200 import focusing

    sc = S.point_target_scene(snr_db=None, seed=11)  # 424 x 512 pulses, 256^2 at 0.08 m, 10 km
    img, fft_ms, bp_ms = O.reference_gpu_focus(sc, reps=1)
    assert fft_ms > 0.0 and bp_ms > 0.0
    with focusing.Plan.for_scene(sc, "fp64") as plan:
        ref64 = plan.focus(sc.phase_history, sc.ant_x, sc.ant_y, sc.ant_z, sc.slant_range, sc.start_freq)[0]
    a = np.abs(img.astype(np.complex128))
    b = np.abs(ref64)
    # the targets focus at the same pixels
    assert np.unravel_index(np.argmax(a), a.shape) == np.unravel_index(np.argmax(b), b.shape)
    # float differential range at 10 km (phase error ~ kr * 1e-3 m) and the
    # roundf bracket make the reference image differ from FP64 by a few tens of
    # percent in relative L2; the magnitude images agree much better
    rel = np.linalg.norm(img - ref64) / np.linalg.norm(ref64)
    rel_mag = np.linalg.norm(a - b) / np.linalg.norm(b)
    assert rel < 1.0 and rel_mag < 0.2, (rel, rel_mag)
