"""lfmm3d_direct_device_noalloc: the direct sum with its source-chunk scratch
in a static device array (no allocation per call), against
lfmm3d_direct_device on the same device buffers.  Two calls in a row with
different sizes: the second reads scratch the first left behind, which must
not matter (nothing in it needs to start at zero)."""
import numpy as np
import pytest

from laplace_fmm_b200.workloads import rel_l2

pytestmark = pytest.mark.gpu
TOL = 1e-13


def _call(ctx, name, src, q, tgt):
    import torch
    dev = torch.device("cuda", ctx.device)
    d = [torch.from_numpy(np.ascontiguousarray(a)).to(dev) for a in (src, q, tgt)]
    pot = torch.zeros(len(tgt), dtype=torch.float64, device=dev)
    fld = torch.zeros(3 * len(tgt), dtype=torch.float64, device=dev)
    torch.cuda.synchronize(dev)
    st = getattr(ctx.lib, name)(ctx.handle, len(src), d[0].data_ptr(), d[1].data_ptr(), len(tgt), d[2].data_ptr(),
                                pot.data_ptr(), fld.data_ptr())
    ctx.check(st, name)
    torch.cuda.ExternalStream(ctx.stream, device=dev).synchronize()
    return pot.cpu().numpy(), fld.cpu().numpy().reshape(-1, 3)


def test_noalloc_matches_direct_device_two_calls(ctx):
    g = np.random.default_rng(5)
    cases = [(200000, 4096), (50000, 300)]
    for ns, nt in cases:
        src = g.random((ns, 3)); q = g.uniform(-1, 1, ns); tgt = g.random((nt, 3))
        pa, fa = _call(ctx, "lfmm3d_direct_device_noalloc", src, q, tgt)
        pb, fb = _call(ctx, "lfmm3d_direct_device", src, q, tgt)
        assert rel_l2(pa, pb) < TOL and rel_l2(fa, fb) < TOL


def test_noalloc_at_the_target_limit(ctx):
    """65,536 targets: the scratch bound (8 MiB / (4 doubles x targets) = 4
    source chunks) is what limits the split here, not the GPU's size."""
    g = np.random.default_rng(11)
    ns, nt = 400000, 65536
    src = g.random((ns, 3)); q = g.uniform(-1, 1, ns); tgt = g.random((nt, 3))
    pa, fa = _call(ctx, "lfmm3d_direct_device_noalloc", src, q, tgt)
    pb, fb = _call(ctx, "lfmm3d_direct_device", src, q, tgt)
    assert rel_l2(pa, pb) < TOL and rel_l2(fa, fb) < TOL


def test_noalloc_allocates_nothing(ctx):
    """What the entry point exists for: after its first call on the device,
    a call leaves the device's free memory (cudaMemGetInfo) unchanged, both
    when it splits the sources (the chunk reduction runs) and when not."""
    import torch
    dev = torch.device("cuda", ctx.device)
    g = np.random.default_rng(12)
    bufs = []
    for ns, nt in [(300000, 2048), (300, 60000)]:
        d = [torch.from_numpy(a).to(dev) for a in (g.random((ns, 3)), g.uniform(-1, 1, ns), g.random((nt, 3)))]
        bufs.append((ns, nt, d, torch.empty(nt, dtype=torch.float64, device=dev),
                     torch.empty(3 * nt, dtype=torch.float64, device=dev)))
    stream = torch.cuda.ExternalStream(ctx.stream, device=dev)

    def call(b):
        ns, nt, d, pot, fld = b
        ctx.check(ctx.lib.lfmm3d_direct_device_noalloc(ctx.handle, ns, d[0].data_ptr(), d[1].data_ptr(), nt,
                                                       d[2].data_ptr(), pot.data_ptr(), fld.data_ptr()), "noalloc")
        stream.synchronize()

    call(bufs[0])                     # the first call on the device sets up (address, kernels)
    torch.cuda.synchronize(dev)
    for b in bufs + bufs:
        free0, _ = torch.cuda.mem_get_info(dev)
        call(b)
        free1, _ = torch.cuda.mem_get_info(dev)
        assert free1 == free0, (b[0], b[1], free0 - free1)


def test_noalloc_rejects_too_many_targets(ctx):
    st = ctx.lib.lfmm3d_direct_device_noalloc(ctx.handle, 10, None, None, 65537, None, None, None)
    assert st == -1
    assert "65536" in ctx.lib.lfmm_last_error(ctx.handle).decode()
