"""Python binding of librav2d_gpu.so, the B200 in-loop filter library.

Mirrors the reference's per-frame filter entry points: `filter_frame`
stands for looping `filter_sbrow` (decode.rs:3718) over a frame and `grain`
for `apply_grain_to_picture_mt` (decode.rs:4672).  The CUDA library is the
only implementation: if it is missing this module raises at import-time use.
"""
import ctypes as C
import os

import numpy as np

from . import abi

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "librav2d_gpu.so")
_lib = None

SYMBOLS = [
    "r2g_version", "r2g_plane_geometry", "r2g_struct_sizes", "r2g_ctx_create", "r2g_ctx_destroy",
    "r2g_last_error", "r2g_frame_alloc", "r2g_frame_free", "r2g_frame_upload_recon", "r2g_frame_filter",
    "r2g_frame_grain", "r2g_download", "r2g_sync", "r2g_filter_frame_host", "r2g_batch_submit", "r2g_wait",
    "r2g_frame_stage", "r2g_frame_run", "r2g_ctx_set_stream", "r2g_ctx_profile", "r2g_ctx_profile_read",
    "r2g_ctx_launch_count", "r2g_film_grain_apply_noalloc", "r2g_batch_config", "r2g_batch_tile_rows", "r2g_server_create",
    "r2g_server_submit", "r2g_server_wait", "r2g_server_close_stream", "r2g_server_stats", "r2g_server_destroy",
    "r2g_ctx_overlap_copies", "r2g_ctx_fence", "r2g_download_y4m", "r2g_y4m_frame_bytes", "r2g_y4m_header",
    "r2g_download_rows", "r2g_dsp_cdef_dir", "r2g_dsp_cdef_filter", "r2g_dsp_ccso_prep", "r2g_dsp_ccso_add",
    "r2g_dsp_gdf_add", "r2g_dsp_generate_grain", "r2g_dsp_ns_wiener_single_y", "r2g_dsp_ns_wiener_single_uv",
    "r2g_dsp_ns_wiener_multi", "r2g_dsp_pc_wiener", "r2g_dsp_gdf_prep", "r2g_ctx_device_faults",
    "r2g_frame_read_masks", "r2g_dsp_deblock_sb64", "r2g_dsp_fgy_32x32xn", "r2g_dsp_fguv_32x32xn",
]


class R2gError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"rav2d_gpu error {code}: {msg}")
        self.code = code


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is not built; run __graft_entry__.build()")
        L = C.CDLL(LIB_PATH)
        L.r2g_last_error.restype = C.c_char_p
        L.r2g_last_error.argtypes = [C.c_void_p]
        L.r2g_ctx_create.argtypes = [C.c_int, C.c_int64, C.POINTER(C.c_void_p)]
        L.r2g_ctx_destroy.argtypes = [C.c_void_p]
        L.r2g_frame_alloc.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_void_p)]
        L.r2g_frame_free.argtypes = [C.c_void_p, C.c_void_p]
        L.r2g_frame_upload_recon.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p,
                                             C.c_int64]
        L.r2g_frame_filter.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(abi.FrameParams),
                                       C.POINTER(abi.SideInfo), C.c_uint32]
        L.r2g_frame_grain.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(abi.FilmGrainData), C.c_uint32]
        L.r2g_download.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p,
                                   C.c_int64]
        L.r2g_sync.argtypes = [C.c_void_p]
        L.r2g_batch_submit.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.POINTER(C.c_uint64)]
        L.r2g_wait.argtypes = [C.c_void_p, C.c_uint64, C.c_int]
        L.r2g_plane_geometry.argtypes = [C.c_int, C.c_int, C.c_int] + [C.POINTER(C.c_int64)] * 4
        L.r2g_struct_sizes.argtypes = [C.POINTER(C.c_int32), C.c_int]
        L.r2g_frame_stage.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(abi.FrameParams), C.POINTER(abi.SideInfo),
                                      C.c_uint32]
        L.r2g_frame_run.argtypes = [C.c_void_p, C.c_void_p]
        L.r2g_frame_read_masks.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]
        L.r2g_ctx_set_stream.argtypes = [C.c_void_p, C.c_void_p]
        L.r2g_ctx_profile.argtypes = [C.c_void_p, C.c_int]
        L.r2g_ctx_profile_read.argtypes = [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int64), C.c_int]
        L.r2g_ctx_device_faults.argtypes = [C.c_void_p, C.POINTER(C.c_uint32)]
        L.r2g_ctx_launch_count.argtypes = [C.c_void_p]
        L.r2g_ctx_launch_count.restype = C.c_int64
        L.r2g_batch_config.argtypes = [C.c_void_p, C.POINTER(C.c_int32), C.c_int]
        L.r2g_batch_tile_rows.argtypes = [C.c_void_p, C.POINTER(C.c_int32), C.c_int]
        L.r2g_server_create.argtypes = [C.c_void_p, C.POINTER(abi.ServeConfig), C.POINTER(C.c_void_p)]
        L.r2g_server_submit.argtypes = [C.c_void_p, C.POINTER(abi.ServeRequest), C.POINTER(C.c_uint64)]
        L.r2g_server_wait.argtypes = [C.c_void_p, C.c_uint64, C.c_int, C.POINTER(abi.ServeResult)]
        L.r2g_server_close_stream.argtypes = [C.c_void_p, C.c_int32]
        L.r2g_server_stats.argtypes = [C.c_void_p, C.POINTER(abi.ServeStats), C.c_int]
        L.r2g_server_destroy.argtypes = [C.c_void_p]
        L.r2g_ctx_overlap_copies.argtypes = [C.c_void_p, C.c_int]
        L.r2g_ctx_fence.argtypes = [C.c_void_p]
        L.r2g_download_y4m.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int64]
        L.r2g_y4m_frame_bytes.argtypes = [C.c_int, C.c_int, C.c_int]
        L.r2g_y4m_frame_bytes.restype = C.c_int64
        vp, i64, ci = C.c_void_p, C.c_int64, C.c_int
        L.r2g_dsp_cdef_dir.argtypes = [vp, i64, C.POINTER(C.c_uint32), ci]
        L.r2g_dsp_cdef_filter.argtypes = [vp, i64, vp, vp, vp] + [ci] * 8
        L.r2g_dsp_ccso_prep.argtypes = [vp, i64, vp, i64, vp, vp, vp] + [ci] * 11
        L.r2g_dsp_ccso_add.argtypes = [vp, i64, vp, i64, vp, vp, ci, ci, vp, ci]
        L.r2g_dsp_gdf_add.argtypes = [vp, i64, vp, i64, ci, ci, ci, vp, ci]
        L.r2g_dsp_generate_grain.argtypes = [vp, vp, vp, C.POINTER(abi.FilmGrainData), C.c_uint32, ci]
        wp = C.POINTER(abi.WienerParams)
        for n in ("r2g_dsp_ns_wiener_single_y", "r2g_dsp_ns_wiener_single_uv", "r2g_dsp_ns_wiener_multi",
                  "r2g_dsp_pc_wiener"):
            getattr(L, n).argtypes = [vp, i64, vp, vp, vp, ci, ci, wp, ci, vp, ci]
        L.r2g_dsp_gdf_prep.argtypes = [vp, i64, vp, i64, vp, vp, vp] + [ci] * 6
        L.r2g_dsp_deblock_sb64.argtypes = [vp, i64, vp, vp, vp, vp] + [ci] * 4
        fgp = C.POINTER(abi.FilmGrainData)
        L.r2g_dsp_fgy_32x32xn.argtypes = [vp, vp, i64, fgp, C.c_uint32, ci, vp, vp, ci, ci, ci]
        L.r2g_dsp_fguv_32x32xn.argtypes = [vp, vp, i64, fgp, C.c_uint32, ci, vp, vp, ci, ci, vp, i64] + [ci] * 5
        L.r2g_y4m_header.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_char_p, C.c_int]
        L.r2g_download_rows.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_int64,
                                        C.c_void_p, C.c_void_p, C.c_int64]
        _lib = L
    return _lib


def _ptr(a):
    return C.c_void_p(a.ctypes.data)


class Context:
    """One device context (streams, tables, memory budget)."""

    def __init__(self, device=0, mem_budget=0):
        h = C.c_void_p()
        rc = lib().r2g_ctx_create(device, mem_budget, C.byref(h))
        if rc != 0:
            raise R2gError(rc, "context creation failed")
        self.h = h

    def check(self, rc):
        if rc != 0:
            raise R2gError(rc, lib().r2g_last_error(self.h).decode())
        return rc

    def sync(self):
        self.check(lib().r2g_sync(self.h))

    def close(self):
        if self.h:
            lib().r2g_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream_handle):
        """Enqueue on a caller-owned cudaStream_t (an int handle; 0 = own)."""
        self.check(lib().r2g_ctx_set_stream(self.h, C.c_void_p(stream_handle or None)))

    def overlap_copies(self, enable=True):
        """Uploads / downloads on their own streams, overlapping kernels."""
        self.check(lib().r2g_ctx_overlap_copies(self.h, int(enable)))

    def fence(self):
        """Make the context stream wait for every copy issued so far."""
        self.check(lib().r2g_ctx_fence(self.h))

    def profile(self, enable=True):
        self.check(lib().r2g_ctx_profile(self.h, int(enable)))

    STAGES = ("deblock", "cdef_ccso", "loop_restoration", "film_grain")

    def profile_read(self):
        ms = (C.c_double * 4)()
        n = (C.c_int64 * 4)()
        self.check(lib().r2g_ctx_profile_read(self.h, ms, n, 4))
        return {s: (ms[i], n[i]) for i, s in enumerate(self.STAGES)}

    def launch_count(self):
        return lib().r2g_ctx_launch_count(self.h)

    def device_faults(self):
        """Bounded device-side waits that ran out so far (0 when healthy)."""
        n = C.c_uint32()
        self.check(lib().r2g_ctx_device_faults(self.h, C.byref(n)))
        return n.value

    def frame(self, width, height, bitdepth):
        return Frame(self, width, height, bitdepth)

    def batch_submit(self, items, staged=False):
        """items: list of (Frame, SynthFrame-like with fp/side()/inloop/fgd/grain_seed).
        staged=True runs every frame with its last Frame.stage() side-info."""
        arr = (abi.BatchItem * len(items))()
        keep = []
        for i, (fr, sf) in enumerate(items):
            arr[i].frame = fr.h
            if not staged:
                side = sf.side()
                keep.append(side)
                arr[i].fp = C.pointer(sf.fp)
                arr[i].side = C.pointer(side)
                arr[i].inloop_mask = sf.inloop
            arr[i].fgd = C.pointer(sf.fgd) if sf.fgd is not None else None
            arr[i].grain_seed = sf.grain_seed
        t = C.c_uint64()
        self.check(lib().r2g_batch_submit(self.h, C.cast(arr, C.c_void_p), len(items), C.byref(t)))
        return t.value

    def wait(self, ticket, timeout_ms=-1):
        return lib().r2g_wait(self.h, C.c_uint64(ticket), timeout_ms)

    def batch_config(self):
        """(SM count, CTAs per SM of the last batch per stage; 0 = one CTA per item)."""
        v = (C.c_int32 * 4)()
        sms = lib().r2g_batch_config(self.h, v, 4)
        return sms, dict(zip(("deblock", "cdef_ccso", "loop_restoration", "film_grain"), list(v)))

    def batch_tile_rows(self):
        """Luma rows per work item of the last batch per stage (the tile shape)."""
        v = (C.c_int32 * 4)()
        lib().r2g_batch_tile_rows(self.h, v, 4)
        return dict(zip(("deblock", "cdef_ccso", "loop_restoration", "film_grain"), list(v)))


class Frame:
    """A device-resident frame: recon, filtered and display buffers."""

    def __init__(self, ctx, width, height, bitdepth):
        self.ctx = ctx
        h = C.c_void_p()
        ctx.check(lib().r2g_frame_alloc(ctx.h, width, height, bitdepth, C.byref(h)))
        self.h = h
        self.width, self.height, self.bitdepth = width, height, bitdepth
        self.dtype = np.uint16 if bitdepth > 8 else np.uint8

    def free(self):
        if self.h:
            lib().r2g_frame_free(self.ctx.h, self.h)
            self.h = None

    def upload(self, planes):
        y, u, v = planes
        self.ctx.check(lib().r2g_frame_upload_recon(self.ctx.h, self.h, _ptr(y), y.strides[0], _ptr(u), _ptr(v),
                                                    u.strides[0]))

    def stage(self, sf, inloop=None):
        side = sf.side()
        self._side = side
        self.ctx.check(lib().r2g_frame_stage(self.ctx.h, self.h, C.byref(sf.fp), C.byref(side),
                                             sf.inloop if inloop is None else inloop))

    def run(self):
        self.ctx.check(lib().r2g_frame_run(self.ctx.h, self.h))

    def read_masks(self):
        """The staged SB256 records as the stage kernels read them."""
        n = ((self.width // 4 + 63) >> 6) * ((self.height // 4 + 63) >> 6)
        out = np.zeros(n, abi.AV2_FILTER_DTYPE)
        self.ctx.check(lib().r2g_frame_read_masks(self.ctx.h, self.h, _ptr(out), n))
        return out

    def download_into(self, out, which=0):
        """Enqueue a download into preallocated (ideally pinned) planes."""
        self.ctx.check(lib().r2g_download(self.ctx.h, self.h, which, _ptr(out[0]), out[0].strides[0],
                                          _ptr(out[1]), _ptr(out[2]), out[1].strides[0]))

    def filter(self, sf, inloop=None):
        side = sf.side()
        self._side = side
        self.ctx.check(lib().r2g_frame_filter(self.ctx.h, self.h, C.byref(sf.fp), C.byref(side),
                                              sf.inloop if inloop is None else inloop))

    def download_y4m(self, which=0, out_bitdepth=0):
        """One Y4M frame ("FRAME\\n" + packed planes) as bytes."""
        n = lib().r2g_y4m_frame_bytes(self.width, self.height, out_bitdepth or self.bitdepth)
        buf = np.zeros(n, np.uint8)
        self.ctx.check(lib().r2g_download_y4m(self.ctx.h, self.h, which, out_bitdepth, _ptr(buf), n))
        self.ctx.sync()
        return buf.tobytes()

    def download_rows(self, like, row0, nrows, which=0):
        """Rows [row0, row0 + nrows) (and the chroma rows under them)."""
        out = [np.zeros((nrows >> (i > 0), p.shape[1]), p.dtype) for i, p in enumerate(like)]
        self.ctx.check(lib().r2g_download_rows(self.ctx.h, self.h, which, row0, nrows, _ptr(out[0]),
                                               out[0].strides[0], _ptr(out[1]), _ptr(out[2]), out[1].strides[0]))
        self.ctx.sync()
        return out

    def grain(self, fgd, seed):
        self.ctx.check(lib().r2g_frame_grain(self.ctx.h, self.h, C.byref(fgd), seed))

    def download(self, like, which=0):
        out = [np.zeros_like(p) for p in like]
        self.ctx.check(lib().r2g_download(self.ctx.h, self.h, which, _ptr(out[0]), out[0].strides[0],
                                          _ptr(out[1]), _ptr(out[2]), out[1].strides[0]))
        self.ctx.sync()
        return out


def filter_frame(ctx, sf, grain=False):
    """Upload, filter (and optionally grain) one SynthFrame; returns the
    filtered planes (and the display planes when grain=True)."""
    fr = Frame(ctx, sf.width, sf.height, sf.bitdepth)
    try:
        fr.upload(sf.planes)
        fr.filter(sf)
        out = fr.download(sf.planes, 0)
        if grain:
            fr.grain(sf.fgd, sf.grain_seed)
            g = fr.download(sf.planes, 1)
            return out, g
        return out
    finally:
        fr.free()


class Server:
    """Continuous-batching server over one context (r2g_server_*)."""

    def __init__(self, ctx, mem_budget=0, max_batch=64, frames_per_stream=2):
        self.ctx = ctx
        cfg = abi.ServeConfig(mem_budget, max_batch, frames_per_stream)
        h = C.c_void_p()
        ctx.check(lib().r2g_server_create(ctx.h, C.byref(cfg), C.byref(h)))
        self.h = h
        self._keep = {}

    def submit(self, stream_id, sf, src, dst, ref=None, grain=True):
        """src/dst/ref: [y, u, v] host arrays (the allocator geometry); the
        arrays and sf's side-info must stay alive until wait()."""
        side = sf.side()
        r = abi.ServeRequest()
        r.stream_id = stream_id
        r.fp = C.pointer(sf.fp)
        r.side = C.pointer(side)
        r.inloop_mask = sf.inloop
        r.fgd = C.pointer(sf.fgd) if (grain and sf.fgd is not None) else None
        r.grain_seed = sf.grain_seed
        r.src_y, r.src_u, r.src_v = (p.ctypes.data for p in src)
        r.src_y_stride, r.src_uv_stride = src[0].strides[0], src[1].strides[0]
        r.dst_y, r.dst_u, r.dst_v = (p.ctypes.data for p in dst)
        r.dst_y_stride, r.dst_uv_stride = dst[0].strides[0], dst[1].strides[0]
        if ref is not None:
            r.ref_y, r.ref_u, r.ref_v = (p.ctypes.data for p in ref)
        i = C.c_uint64()
        self.ctx.check(lib().r2g_server_submit(self.h, C.byref(r), C.byref(i)))
        self._keep[i.value] = (side, r, src, dst, ref)
        return i.value

    def wait(self, rid, timeout_ms=-1):
        """Returns (rc, ServeResult); rc is the wait's own status."""
        res = abi.ServeResult()
        rc = lib().r2g_server_wait(self.h, C.c_uint64(rid), timeout_ms, C.byref(res))
        if rc == 0:
            self._keep.pop(rid, None)
        return rc, res

    def close_stream(self, stream_id):
        return lib().r2g_server_close_stream(self.h, stream_id)

    def stats(self, reset=False):
        st = abi.ServeStats()
        self.ctx.check(lib().r2g_server_stats(self.h, C.byref(st), int(reset)))
        return {k: getattr(st, k) for k, _ in abi.ServeStats._fields_}

    def close(self):
        if self.h:
            lib().r2g_server_destroy(self.h)
            self.h = None
            self._keep.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def y4m_header(width, height, fps_num, fps_den, bitdepth):
    buf = C.create_string_buffer(128)
    n = lib().r2g_y4m_header(width, height, fps_num, fps_den, bitdepth, buf, 128)
    if n < 0:
        raise R2gError(n, "bad Y4M header parameters")
    return buf.raw[:n]
