"""ctypes front-end of the CPU oracle (oracle/_build/liboracle.so).

TEST INFRASTRUCTURE ONLY: the parity tests, the smoke check and the
benchmark's CPU-baseline leg use this to compute the reference's filter
output on the CPU.  The product library never imports it.
"""
import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None


def build():
    subprocess.check_call(["make", "-s", "-j8"], cwd=_HERE)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = C.CDLL(_LIB_PATH)
        _lib.r2o_filter_frame.restype = C.c_int
        _lib.r2o_apply_grain.restype = C.c_int
        _lib.r2o_deblock_quant_thr.restype = C.c_uint32
        _lib.r2o_deblock_side_thr.restype = C.c_uint32
        _lib.r2o_ccso_score.restype = C.c_uint32
        _lib.r2o_get_random_number.restype = C.c_uint32
    return _lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def filter_frame(sf, inloop=None):
    """Run the reference's per-sbrow filter pass over a SynthFrame; returns
    the filtered [y, u, v] planes in the frame's own sample dtype."""
    from rav2d_b200 import abi  # noqa: F401  (ctypes structs)
    planes16 = [np.ascontiguousarray(p.astype(np.uint16)) for p in sf.planes]
    side = sf.side()
    rc = lib().r2o_filter_frame(C.byref(sf.fp), C.byref(side), C.c_uint32(sf.inloop if inloop is None else inloop),
                                _p(planes16[0]), _p(planes16[1]), _p(planes16[2]),
                                C.c_int64(planes16[0].shape[1]), C.c_int64(planes16[1].shape[1]))
    if rc != 0:
        raise ValueError("oracle rejected the frame")
    dt = sf.planes[0].dtype
    return [p.astype(dt) for p in planes16]


def build_db_masks(sf):
    """The frame's edge masks from its block records (SynthFrame.use_db_blocks),
    walked in decode order as the decoder's create_db_mask calls do; returns a
    copy of sf.masks with filter_y / filter_uv rebuilt."""
    masks = sf.masks.copy()
    lib().r2o_build_db_masks(C.byref(sf.meta["db_input"]), C.byref(sf.fp), _p(masks), C.c_int(masks.shape[0]))
    return masks


def apply_grain(sf, planes):
    """Film grain on filtered planes; returns the display-copy planes."""
    src = [np.ascontiguousarray(p.astype(np.uint16)) for p in planes]
    dst = [np.zeros_like(p) for p in src]
    lib().r2o_apply_grain(C.byref(sf.fgd), C.c_uint32(sf.grain_seed), sf.width, sf.height, sf.bitdepth,
                          _p(src[0]), _p(src[1]), _p(src[2]), _p(dst[0]), _p(dst[1]), _p(dst[2]),
                          C.c_int64(src[0].shape[1]), C.c_int64(src[1].shape[1]))
    dt = planes[0].dtype
    return [p.astype(dt) for p in dst]


def prep_grain(fgd, seed, bitdepth):
    luts = [np.zeros((73, 82), np.int16) for _ in range(3)]
    scal = [np.zeros(4096, np.uint8) for _ in range(3)]
    lib().r2o_prep_grain(C.byref(fgd), C.c_uint32(seed), bitdepth, _p(luts[0]), _p(luts[1]), _p(luts[2]),
                         _p(scal[0]), _p(scal[1]), _p(scal[2]))
    return luts, [s[:1 << bitdepth] for s in scal]
