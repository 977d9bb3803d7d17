"""Output formatting (Y4M frames packed on the device) and row-band downloads.

The Y4M frame must be byte-identical to what rav2d-cli writes for the same
picture (FRAME marker, then the tightly packed planes, little-endian 16-bit
samples above 8 bits), built here from the regular download; the optional
8-bit display reduction must equal (v + 2) >> 2 clipped; a row band must
equal the same rows of the whole-frame download."""
import numpy as np
import pytest

from rav2d_b200 import synth


def _packed(planes, sf, dtype):
    w, h = sf.width, sf.height
    parts = [planes[0][:h, :w], planes[1][:h // 2, :w // 2], planes[2][:h // 2, :w // 2]]
    return b"FRAME\n" + b"".join(np.ascontiguousarray(p).astype(dtype).tobytes() for p in parts)


def test_y4m_header_matches_cli_format():
    from rav2d_b200 import gpu

    assert gpu.y4m_header(1920, 1080, 30, 1, 10) == b"YUV4MPEG2 W1920 H1080 F30:1 Ip C420p10\n"
    assert gpu.y4m_header(640, 360, 25, 1, 8) == b"YUV4MPEG2 W640 H360 F25:1 Ip C420jpeg\n"


@pytest.mark.gpu
@pytest.mark.parametrize("bd", [8, 10])
def test_y4m_and_rows_match_download(bd):
    from rav2d_b200 import gpu

    sf = synth.make_frame(640, 360, bd, 0x0A4F0000 + bd, chain="full", grain=True)
    ctx = gpu.Context(0)
    try:
        fr = ctx.frame(sf.width, sf.height, bd)
        fr.upload(sf.planes)
        fr.filter(sf)
        fr.grain(sf.fgd, sf.grain_seed)
        filt = fr.download(sf.planes, 0)
        disp = fr.download(sf.planes, 1)
        dt = "<u2" if bd > 8 else "u1"
        assert fr.download_y4m(0) == _packed(filt, sf, dt)
        assert fr.download_y4m(1) == _packed(disp, sf, dt)
        if bd == 10:
            red = [np.minimum((p.astype(np.int32) + 2) >> 2, 255) for p in disp]
            assert fr.download_y4m(1, out_bitdepth=8) == _packed(red, sf, "u1")
        rows = fr.download_rows(sf.planes, 64, 100, which=0)
        assert np.array_equal(rows[0][:, :sf.width], filt[0][64:164, :sf.width])
        for pl in (1, 2):
            assert np.array_equal(rows[pl][:, :sf.width // 2], filt[pl][32:82, :sf.width // 2])
        fr.free()
    finally:
        ctx.close()
