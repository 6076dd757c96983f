"""The kernels' u8 -> float conversion: with x = i / 256 (exact), one fused
multiply-add fma(x, fl(1/255), x) equals the correctly rounded i / 255 (the
reference's frame reader, ffmpeg_io.c:293) for every byte value.  The FMA is
evaluated exactly in double precision here (x has 8 significant bits and
fl(1/255) 24, so x*c + x is exact in double) and rounded once to float, which
is what the device's fused multiply-add does."""
import numpy as np


def test_u8_to_float_by_fma_is_correctly_rounded():
    i = np.arange(256)
    want = (i.astype(np.float32) / np.float32(255)).astype(np.float32)
    c = np.float64(np.float32(1.0) / np.float32(255.0))
    x = i.astype(np.float64) / 256.0
    got = (x * c + x).astype(np.float32)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
