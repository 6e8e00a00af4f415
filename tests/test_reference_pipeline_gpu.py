"""End-to-end parity of the drop-in modules with the reference's interpolated-mode tail.

image_processor.py:383-396 with its imports swapped to mmnorm_b200's image_cuda and
normal_estimates_cuda, against the same calls run the reference's way: its own CUDA
kernels (compiled unmodified from the reference's sources) behind its host steps
(oracle/ref_pipeline.py).  Both sides take the same numpy range FFT.  The bit-exact form
must reproduce the reference's image and unit normals bit for bit (antenna counts are
powers of two here, so the per-group mean divides exactly in either precision); the fast
form within the tolerances of its own tests.  Monostatic, four RX offsets with the
use_4_rx re-layout, and the TI radar's 0.15 m range offset."""
import numpy as np
import pytest

from mmnorm_b200 import scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ref_pipeline():
    from oracle import ref_cuda
    if not ref_cuda.available():
        pytest.skip("reference kernels not built (oracle/build.py)")
    from oracle import ref_pipeline
    return ref_pipeline


def _case(rx, is_ti):
    sc = scenes.sphere_scene(seed=70 + rx + 2 * is_ti, n_ap=32 if rx == 1 else 16, nf=64,
                             n_vox=24, n_pts=60)
    A, S = sc.meas.shape
    rng = np.random.default_rng(71)
    if rx == 1:
        radar = sc.meas.reshape(A, S, 1)
        rxo = np.zeros((1, 3), np.float32)
    else:
        rxo = np.array([[0, -0.002, 0], [0, -0.004, 0], [0, -0.006, 0], [0, -0.008, 0]],
                       np.float32)
        noise = (rng.standard_normal((A, S, rx)) + 1j * rng.standard_normal((A, S, rx))) * 0.05
        radar = (sc.meas[:, :, None] + noise).astype(np.complex64)
    return sc, np.ascontiguousarray(radar), rxo


@pytest.mark.parametrize("rx,is_ti", [(1, 0), (4, 0), (1, 1)])
def test_dropin_tail_matches_reference(cuda_dev, ref_pipeline, rx, is_ti):
    from mmnorm_b200 import py_image_gpu, py_sn_est_gpu
    sc, radar, rxo = _case(rx, is_ti)
    A, S, R = radar.shape
    locs = np.asarray(sc.antenna_locs, np.float32)
    wl, sl, bw = np.float32(sc.wavelength), np.float32(sc.slope), sc.f_hi - sc.f_lo
    bins = ref_pipeline.range_fft_host(radar, 4096)
    img_r, nrm_r = ref_pipeline.reference_dropin_calls(sc.x_locs, sc.y_locs, sc.z_locs, locs,
                                                       bins, rxo, sl, wl, bw, S, is_ti)
    for precision in ("exact", "fast"):
        img, _ = py_image_gpu.image_cuda(sc.x_locs, sc.y_locs, sc.z_locs, locs, bins, rxo,
                                         float(sl), float(wl), bw, S, use_4_rx=True,
                                         is_ti_radar=bool(is_ti),
                                         use_interpolated_processing=True, precision=precision)
        nrm = py_sn_est_gpu.normal_estimates_cuda(img, sc.x_locs, sc.y_locs, sc.z_locs, locs,
                                                  bins, rxo, float(sl), float(wl), bw, S,
                                                  use_4_rx=True, is_ti_radar=bool(is_ti),
                                                  precision=precision)
        nrm /= np.linalg.norm(nrm, axis=-1)[..., np.newaxis].repeat(3, axis=-1)
        fin_o, fin_r = np.isfinite(nrm).all(-1), np.isfinite(nrm_r).all(-1)
        if precision == "exact":
            assert np.array_equal(img.astype(np.complex128), img_r)
            assert np.array_equal(fin_o, fin_r)
            assert np.array_equal(nrm[fin_o], nrm_r[fin_r])
        else:
            rel = np.linalg.norm(img - img_r) / np.linalg.norm(img_r)
            assert rel < 2e-6, rel
            assert np.mean(fin_o == fin_r) > 0.999
            both = fin_o & fin_r
            cosang = np.clip(np.sum(nrm[both] * nrm_r[both], axis=-1), -1.0, 1.0)
            assert np.median(np.degrees(np.arccos(cosang))) < 1e-3


@pytest.mark.parametrize("rx,is_ti", [(1, 0), (4, 1)])
def test_dropin_full_mode_image_matches_reference(cuda_dev, ref_pipeline, rx, is_ti):
    """Full matched filter through image_cuda: the reference's cuda_image (FP32 range and
    phase, FP64 sin/cos) behind its host steps against the drop-in's mixed-precision
    kernel behind the same contract (/A twice, complex image, phase centres).  The forms
    differ by the reference's FP32 range error (~3e-5 relative; bound 2e-4)."""
    from mmnorm_b200 import py_image_gpu
    sc, radar, rxo = _case(rx, is_ti)
    A, S, R = radar.shape
    locs = np.asarray(sc.antenna_locs, np.float32)
    wl, sl, bw = np.float32(sc.wavelength), np.float32(sc.slope), sc.f_hi - sc.f_lo
    img_r, cen_r = ref_pipeline.reference_full_image(sc.x_locs, sc.y_locs, sc.z_locs, locs,
                                                     radar, rxo, sl, wl, bw, S, is_ti)
    img, cen = py_image_gpu.image_cuda(sc.x_locs, sc.y_locs, sc.z_locs, locs, radar, rxo,
                                       float(sl), float(wl), bw, S, use_4_rx=True,
                                       is_ti_radar=bool(is_ti),
                                       use_interpolated_processing=False)
    rel = np.linalg.norm(img - img_r) / np.linalg.norm(img_r)
    assert rel < 2e-4, rel
    assert np.allclose(cen, cen_r, rtol=0, atol=1e-7)
