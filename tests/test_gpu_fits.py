"""FITS data blocks converted on the device (sexgpu_extract_fits) give the
catalogue, segmentation and subtracted frame that the float frame of the
FITS reader's conversion (restated in oracle.fits_to_float) gives through
sexgpu_extract, for every BITPIX, with BSCALE/BZERO, BLANK and non-finite
pixels."""
import numpy as np
import pytest

import synth
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _block(img, bitpix, seed):
    rng = np.random.default_rng(seed)
    h, w = img.shape
    bad = rng.choice(w * h, 40, replace=False)
    if bitpix == 8:
        fmt = dict(bscale=4.0, bzero=700.0, blank=0)
        v = np.clip(np.round((img - 700.0) / 4.0), 1, 255).astype(">u1").ravel()
        v[bad] = 0
    elif bitpix == 16:
        fmt = dict(bscale=0.5, bzero=800.0, blank=-32768)
        v = np.clip(np.round((img - 800.0) / 0.5), -32767, 32767).astype(">i2").ravel()
        v[bad] = -32768
    elif bitpix == 32:
        fmt = dict(bscale=0.01, bzero=3.0, blank=-2147483648)
        v = np.round((img.astype(np.float64) - 3.0) / 0.01).astype(">i4").ravel()
        v[bad] = -2147483648
    elif bitpix == -32:
        fmt = dict(bscale=2.0, bzero=-5.0)
        v = ((img + 5.0) / 2.0).astype(">f4").ravel()
        v[bad[:20]] = np.nan
        v[bad[20:]] = np.inf
    else:
        fmt = dict(bscale=1.0, bzero=0.0)
        v = (img.astype(np.float64) * 1.000000123).astype(">f8").ravel()
        v[bad] = np.nan
    return v.tobytes(), fmt


@pytest.mark.parametrize("bitpix", [8, 16, 32, -32, -64])
def test_fits_block_on_device(gpu_ctx, bitpix):
    img = synth.frame_c0(seed=41, w=420, h=310, nsrc=400)
    raw, fmt = _block(img, bitpix, 7)
    frame = O.fits_to_float(raw, bitpix, **fmt).reshape(img.shape)
    g1, s1, _, sub1, _ = gpu_ctx.extract_fits(raw, bitpix, 420, 310, want_maps=True, **fmt)
    g2, s2, _, sub2, _ = gpu_ctx.extract(frame, want_maps=True)
    assert len(g1) == len(g2) > 20
    assert g1.tobytes() == g2.tobytes()
    assert np.array_equal(s1, s2)
    assert np.array_equal(sub1, sub2)
    if bitpix < 0 or "blank" in fmt:
        assert (frame <= -1e30).sum() == 40
