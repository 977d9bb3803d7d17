"""The allocation-free film-grain entry point agrees with r2g_frame_grain and
with the oracle.

Callers that cannot call cudaMalloc (a decoder inside a framework that owns
all device memory through its own allocator or a fixed pool, or an output
thread that must not block in the driver's allocator) use
r2g_film_grain_apply_noalloc with their own device buffers; its scratch is a
fixed device array inside the library.  Two calls in a row, on different
frames, must each reproduce the grained display copy of the regular entry
point and of the CPU oracle's film grain sample for sample (the path is
integer arithmetic: tolerance 0).  This file is collected last so a failure
here leaves every other test run.
"""
import ctypes as C

import numpy as np
import pytest

from rav2d_b200 import synth

pytestmark = pytest.mark.gpu


def _noalloc(lib, planes, sf, stream):
    import torch

    dt = torch.int16 if sf.bitdepth > 8 else torch.uint8
    src = [torch.from_numpy(p.view(np.int16) if p.dtype == np.uint16 else p).to(dtype=dt).cuda() for p in planes]
    dst = [torch.zeros_like(t) for t in src]
    bps = 2 if sf.bitdepth > 8 else 1
    # the uploads and zero fills above ran on torch's current stream; the
    # grain kernels run on `stream`
    stream.wait_stream(torch.cuda.current_stream())
    rc = lib.r2g_film_grain_apply_noalloc(
        C.c_void_p(src[0].data_ptr()), C.c_void_p(src[1].data_ptr()), C.c_void_p(src[2].data_ptr()),
        C.c_void_p(dst[0].data_ptr()), C.c_void_p(dst[1].data_ptr()), C.c_void_p(dst[2].data_ptr()),
        C.c_int64(planes[0].shape[1] * bps), C.c_int64(planes[1].shape[1] * bps), sf.width, sf.height,
        sf.bitdepth, C.byref(sf.fgd), C.c_uint32(sf.grain_seed), C.c_void_p(stream.cuda_stream))
    assert rc == 0
    torch.cuda.synchronize()
    out = []
    for t, p in zip(dst, planes):
        a = t.cpu().numpy()
        out.append(a.view(np.uint16) if p.dtype == np.uint16 else a)
    return out


def test_noalloc_grain_matches_frame_grain(oracle):
    import torch

    from rav2d_b200 import gpu

    lib = gpu.lib()
    lib.r2g_film_grain_apply_noalloc.restype = C.c_int
    ctx = gpu.Context(0)
    stream = torch.cuda.Stream()
    try:
        frames = [synth.make_frame(640, 360, 10, 0x5EED00A1, chain="full", grain=True),
                  synth.make_frame(320, 176, 8, 0x5EED00A2, chain="db_cdef", grain=True)]
        g = frames[1].fgd
        g.chroma_scaling_from_luma = 0
        for pl in (1, 2):
            g.num_points[pl] = 3
            for i, (x, y) in enumerate([(16, 40), (128, 90), (240, 20)]):
                g.points[pl][i][0], g.points[pl][i][1] = x, y
            g.uv_mult[pl - 1], g.uv_luma_mult[pl - 1], g.uv_offset[pl - 1] = 37, -50, 12
        for sf in frames:  # two calls in a row
            filtered, want = gpu.filter_frame(ctx, sf, grain=True)
            got = _noalloc(lib, filtered, sf, stream)
            ref = oracle.apply_grain(sf, filtered)
            for pl in range(3):
                h, w = sf.height >> (pl > 0), sf.width >> (pl > 0)
                assert np.array_equal(got[pl][:h, :w], want[pl][:h, :w]), f"plane {pl} differs"
                assert np.array_equal(got[pl][:h, :w], ref[pl][:h, :w]), f"plane {pl} differs from the oracle"
    finally:
        ctx.close()


def test_noalloc_unaligned_planes():
    """Planes that start off a 16-byte boundary, with strides that are not
    multiples of 16 bytes, take the sample-by-sample path of the apply kernel;
    it must agree with the regular entry point (aligned, vector path)."""
    import torch

    from rav2d_b200 import gpu

    lib = gpu.lib()
    lib.r2g_film_grain_apply_noalloc.restype = C.c_int
    ctx = gpu.Context(0)
    stream = torch.cuda.Stream()
    try:
        for sf in (synth.make_frame(328, 136, 8, 0x5EED00A3, chain="db", grain=True),
                   synth.make_frame(200, 72, 10, 0x5EED00A4, chain="db", grain=True)):
            filtered, want = gpu.filter_frame(ctx, sf, grain=True)
            bps = 2 if sf.bitdepth > 8 else 1
            dt = torch.int16 if bps == 2 else torch.uint8
            pad, lead = 3, 1  # samples: 3 past each row, 1 before the plane
            src, dst, strides = [], [], []
            for pl, p in enumerate(filtered):
                h, w = sf.height >> (pl > 0), sf.width >> (pl > 0)
                s = w + pad
                buf = torch.zeros(lead + h * s, dtype=dt, device="cuda")
                rows = torch.from_numpy(np.ascontiguousarray(p[:h, :w]).view(np.int16) if bps == 2 else
                                        np.ascontiguousarray(p[:h, :w])).to(dtype=dt).cuda()
                buf[lead:].view(h, s)[:, :w] = rows
                src.append(buf)
                dst.append(torch.zeros_like(buf))
                strides.append(s * bps)
            ptr = [C.c_void_p(t.data_ptr() + lead * bps) for t in src + dst]
            stream.wait_stream(torch.cuda.current_stream())
            rc = lib.r2g_film_grain_apply_noalloc(*ptr, C.c_int64(strides[0]), C.c_int64(strides[1]), sf.width,
                                                  sf.height, sf.bitdepth, C.byref(sf.fgd), C.c_uint32(sf.grain_seed),
                                                  C.c_void_p(stream.cuda_stream))
            assert rc == 0
            torch.cuda.synchronize()
            for pl in range(3):
                h, w = sf.height >> (pl > 0), sf.width >> (pl > 0)
                got = dst[pl][lead:].view(h, strides[pl] // bps)[:, :w].cpu().numpy()
                if bps == 2:
                    got = got.view(np.uint16)
                assert np.array_equal(got, want[pl][:h, :w]), f"plane {pl} differs"
    finally:
        ctx.close()


def test_noalloc_rejects_oversized_bitdepth():
    from rav2d_b200 import abi, gpu

    lib = gpu.lib()
    sf = synth.make_frame(64, 64, 10, 3, chain="db", grain=True)
    one = C.c_void_p(1)
    rc = lib.r2g_film_grain_apply_noalloc(one, one, one, one, one, one, C.c_int64(256), C.c_int64(128), 64, 64, 12,
                                          C.byref(sf.fgd), C.c_uint32(0), None)
    assert rc == abi.R2G_E_TOO_LARGE


def test_noalloc_rejects_out_of_range_grain_fields():
    """Film-grain fields outside the ranges the reference's parser admits
    (obu.rs:272-325) are rejected before any device work."""
    from rav2d_b200 import abi, gpu

    lib = gpu.lib()
    sf = synth.make_frame(64, 64, 10, 4, chain="db", grain=True)
    one = C.c_void_p(1)
    for field, value in (("num_points", 15), ("ar_coeff_shift", 10), ("grain_scale_shift", 4)):
        fgd = type(sf.fgd).from_buffer_copy(sf.fgd)
        if field == "num_points":
            fgd.num_points[0] = value
        else:
            setattr(fgd, field, value)
        rc = lib.r2g_film_grain_apply_noalloc(one, one, one, one, one, one, C.c_int64(256), C.c_int64(128), 64, 64,
                                              10, C.byref(fgd), C.c_uint32(0), None)
        assert rc == abi.R2G_E_INVALID, field
