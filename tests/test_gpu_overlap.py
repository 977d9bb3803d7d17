"""Copy overlap (r2g_ctx_overlap_copies): uploads and downloads on their own
streams while kernels of other frames run.

A ring of three device frames is reused by twelve consecutive frames without
any host synchronisation in between, so every write-after-read hazard of the
ordering (a new upload over a recon that earlier kernels still read, kernels
over planes a download still reads) is exercised; every output must equal
the same frame filtered with overlap off (tolerance 0: integer path)."""
import numpy as np
import pytest

from rav2d_b200 import synth

pytestmark = pytest.mark.gpu


def _same(a, b, sf, what):
    for pl in range(3):
        h, w = sf.height >> (pl > 0), sf.width >> (pl > 0)
        assert np.array_equal(a[pl][:h, :w], b[pl][:h, :w]), f"{what}: plane {pl} differs"


def test_overlapped_ring_equals_serial():
    from rav2d_b200 import gpu

    import dataclasses

    import torch

    def pinned(a):
        t = torch.empty(a.nbytes, dtype=torch.uint8, pin_memory=True)
        out = t.numpy().view(a.dtype).reshape(a.shape)
        out[...] = a
        return out

    sfs = [synth.make_frame(640, 360, 10, 0x0E41A000 + i, chain="full", grain=i % 2 == 0) for i in range(6)]
    # frames 3..5 carry page-locked side-info, which is uploaded without staging
    sfs = [dataclasses.replace(sf, masks=pinned(sf.masks), lr=pinned(sf.lr)) if i >= 3 else sf
           for i, sf in enumerate(sfs)]
    ctx = gpu.Context(0)
    try:
        want = [gpu.filter_frame(ctx, sf, grain=sf.fgd is not None) for sf in sfs]
        ctx.overlap_copies(True)
        ring = [ctx.frame(640, 360, 10) for _ in range(3)]
        got = []
        for i in range(12):
            sf, fr = sfs[i % 6], ring[i % 3]
            fr.upload(sf.planes)
            fr.stage(sf)
            fr.run()
            f = [np.zeros_like(p) for p in sf.planes]
            fr.download_into(f, 0)
            g = None
            if sf.fgd is not None:
                fr.grain(sf.fgd, sf.grain_seed)
                g = [np.zeros_like(p) for p in sf.planes]
                fr.download_into(g, 1)
            got.append((sf, f, g))
        ctx.sync()
        for i, (sf, f, g) in enumerate(got):
            w = want[i % 6]
            if g is not None:
                _same(f, w[0], sf, f"filtered, step {i}")
                _same(g, w[1], sf, f"grained, step {i}")
            else:
                _same(f, w, sf, f"filtered, step {i}")
        # a batch over the same frames honours the pending copies too
        for k, fr in enumerate(ring):
            fr.upload(sfs[k].planes)
        t = ctx.batch_submit([(fr, sfs[k]) for k, fr in enumerate(ring)])
        assert ctx.wait(t, 60000) == 0
        for k, fr in enumerate(ring):
            f = [np.zeros_like(p) for p in sfs[k].planes]
            fr.download_into(f, 0)
            ctx.sync()
            w = want[k][0] if sfs[k].fgd is not None else want[k]
            _same(f, w, sfs[k], f"batch after overlapped copies, frame {k}")
        for fr in ring:
            fr.free()
    finally:
        ctx.close()
