"""This library's scores against the reference's OWN GPU path on the same
series: FFACUDA<float> / FFACUDA<ComplexTypeCUDA>::execute on device spans and
snr_boxcar_3d_cuda_d (lib/ffa_cuda.cu, lib/score_cuda.cu), built from the
reference checkout by oracle/Makefile (target refgpu) into
oracle/_ref/libloki_ref_cuda.so. Skipped where that library was not built.

The reference's GPU code is FP32 with its own summation orders (and, in the
Fourier domain, cuFFT and fast-math sincos), so the comparison is a
tolerance: S/N within 2e-3 + 1e-4 |S/N| in time, 5e-2 + 5e-3 |S/N| through
the Fourier domain (the reference's merges rotate with __sincosf of phases up
to 2 pi nbins/2; its own CUDA-vs-CPU tests allow 5.0 absolute on the folds).
Bit-exact parity of this library is anchored on the reference's CPU code
(the other GPU tests); this file shows that the two GPU paths agree."""

from __future__ import annotations

import numpy as np
import pytest

from conftest import series
from oracle import ref

pytestmark = pytest.mark.gpu

# name -> (nsamps, tsamp, nbins, eta, param_limits, use_fourier)
CASES = {
    "freq_nb64": (2**18, 64e-6, 64, 1.0, [[5.0, 50.0]], False),
    "accel_nb64": (2**20, 64e-6, 64, 2.0, [[-200.0, 200.0], [5.0, 50.0]], False),
    "fourier_freq_nb64": (2**18, 1e-3, 64, 1.0, [[5.0, 8.0]], True),
    "fourier_accel_nb64": (2**18, 1e-3, 64, 2.0, [[-300.0, 300.0], [5.0, 8.0]], True),
    "fourier_accel_nb64_ts250": (2**18, 2.5e-4, 64, 2.0, [[-100.0, 100.0], [5.0, 20.0]], True),
}
WIDTHS = [1, 2, 3, 4, 6, 9, 14]
TOL = {False: (2e-3, 1e-4), True: (5e-2, 5e-3)}
# The reference's GPU Fourier brute fold is well defined only while a segment
# (e and v, FP32) fits the 48 KB default shared memory of a block: beyond it
# kernel_fold_complex_unified<false> (lib/kernels_cuda.cu) runs its block
# reduction after threads >= nbins_f have returned. Fourier cases stay below.
SHARED_LIMIT = 48 * 1024


@pytest.mark.parametrize("name", sorted(CASES))
def test_scores_match_reference_gpu(cuda, name):
    if not ref.gpu_available():
        pytest.skip("oracle/_ref/libloki_ref_cuda.so not built (make -C oracle refgpu)")
    from loki_b200.configs import PulsarSearchConfig
    from loki_b200.ffa import FFACOMPLEXCUDA, FFACUDA

    torch = cuda
    nsamps, tsamp, nbins, eta, lims, use_fourier = CASES[name]
    ts_e, ts_v = series(nsamps, 23)
    # an injected pulse train so that the top of the S/N range is exercised
    t = np.arange(nsamps) * tsamp
    f0 = 0.37 * lims[-1][0] + 0.63 * lims[-1][1]
    ts_e = ts_e + (np.cos(2 * np.pi * f0 * t) > 0.95).astype(np.float32) * 0.4
    cfg = PulsarSearchConfig(nsamps, tsamp, nbins, eta, np.array(lims), use_fourier=use_fourier,
                             score_widths=WIDTHS)
    e = torch.from_numpy(ts_e.astype(np.float32)).cuda()
    v = torch.from_numpy(ts_v).cuda()
    ffa = (FFACOMPLEXCUDA if use_fourier else FFACUDA)(cfg)
    if use_fourier:
        assert 2 * int(ffa.plan.segment_lens[0]) * 4 <= SHARED_LIMIT
    ours = ffa.scores(e, v).cpu().numpy()

    R = ref.RefGPU(ref.make_cfg(nsamps, tsamp, nbins, eta, lims), device=0, use_fourier=use_fourier)
    fold = torch.empty(R.fold_len, dtype=torch.float32, device="cuda")
    w = torch.tensor(WIDTHS, dtype=torch.int32, device="cuda")
    got = torch.empty(R.ncoords_final * len(WIDTHS), dtype=torch.float32, device="cuda")
    R.scores(e.data_ptr(), v.data_ptr(), nsamps, fold.data_ptr(), w.data_ptr(), len(WIDTHS), got.data_ptr(),
             torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    theirs = got.cpu().numpy()

    assert ours.shape == theirs.shape
    atol, rtol = TOL[use_fourier]
    d = np.abs(ours.astype(np.float64) - theirs)
    bound = atol + rtol * np.abs(theirs)
    assert np.all(np.isfinite(theirs))
    assert np.all(d <= bound), f"{name}: max |d| {d.max():.3g} at S/N {theirs.flat[d.argmax()]:.3g}"
    # the same best candidate
    assert abs(float(ours.max()) - float(theirs.max())) <= atol + rtol * abs(float(theirs.max()))
