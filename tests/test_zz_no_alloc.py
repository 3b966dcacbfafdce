"""The multipole entry point that allocates no device memory.

Some callers cannot call cudaMalloc while they run (a fixed device-memory
budget, threads that must not trigger the implicit device synchronisation of
cudaMalloc/cudaFree, hot-path tasks that use recycled buffers).
otfmm_m2l_soa_host_noalloc serves them from a static device array. This test
calls it twice in a row through the C ABI and checks each result against the
allocating host-buffer entry point otfmm_m2l_soa_host (bit-identical for the
exact form, 1e-12 for the fast form, the tolerances of the other GPU tests),
that the exact form also equals the oracle bit for bit, that a call made after
a warm-up call leaves the device's free memory unchanged, and that a batch
larger than the array is refused.
"""
from __future__ import annotations

import numpy as np
import pytest

from octotiger_b200 import synthetic as syn
from octotiger_b200.layout import DRHODT, NCELL, RHO

pytestmark = pytest.mark.gpu


def _cells(a, ncomp):
    return np.asarray(a).reshape(ncomp, -1)[:, :NCELL]


def test_noalloc_matches_allocating_entry_point(oracle):
    from octotiger_b200.otfmm import Context, OtfmmError
    ctx = Context(0, 0.5)
    try:
        # call 1: two refined subgrids, RHO, exact FP64
        staged = []
        for seed, leaf_dirs in ((61, ()), (62, (1, 5, 20))):
            b = syn.single_subgrid(seed=seed, leaf_dirs=leaf_dirs)
            staged.append(oracle.stage_m2l(b.pool, b.items[0]))
        mon = np.stack([s[0] for s in staged])
        M = np.stack([s[1] for s in staged])
        com = np.stack([s[2] for s in staged])
        L, Lc = ctx.m2l_soa_host_noalloc(mon, M, com, RHO, False, "fp64_exact")
        for i in range(2):
            Lr, Lcr = ctx.m2l_soa_host(mon[i], M[i], com[i], RHO, False, "fp64_exact")
            np.testing.assert_array_equal(_cells(L[i], 20), _cells(Lr, 20))
            np.testing.assert_array_equal(_cells(Lc[i], 3), _cells(Lcr, 3))
            Lo, Lco = oracle.m2l_soa(0.5, mon[i], M[i], com[i], rho=True, root=False)
            np.testing.assert_array_equal(_cells(L[i], 20), _cells(Lo, 20))
            np.testing.assert_array_equal(_cells(Lc[i], 3), _cells(Lco, 3))
        # call 2 right after: the root stencil, DRHODT, fast FP64
        r = syn.root_subgrid(seed=63)
        _, Mr, comr = oracle.stage_m2l(r.pool, r.items[0])
        L2, _ = ctx.m2l_soa_host_noalloc(None, Mr[None], comr[None], DRHODT, True, "fp64")
        Lr2, _ = ctx.m2l_soa_host(None, Mr, comr, DRHODT, True, "fp64")
        got, ref = _cells(L2[0], 20), _cells(Lr2, 20)
        scale = np.abs(ref).max(axis=1)
        assert (np.abs(got - ref).max(axis=1) <= 1e-12 * scale).all()
        # the call allocates nothing: the device's free memory is the same
        # before and after a call that follows a warm-up call
        import torch
        ctx.m2l_soa_host_noalloc(mon, M, com, RHO, False, "fp64")   # warm-up: loads this kernel
        free0, _ = torch.cuda.mem_get_info(0)
        L3, _ = ctx.m2l_soa_host_noalloc(mon, M, com, RHO, False, "fp64")
        free1, _ = torch.cuda.mem_get_info(0)
        assert free1 == free0, (free0, free1)
        Lf, _ = ctx.m2l_soa_host(mon[1], M[1], com[1], RHO, False, "fp64")
        scale = np.abs(_cells(Lf, 20)).max(axis=1)
        assert (np.abs(_cells(L3[1], 20) - _cells(Lf, 20)).max(axis=1) <= 1e-12 * scale).all()
        # more subgrids than the static array holds: refused, nothing run
        with pytest.raises(OtfmmError) as e:
            ctx.m2l_soa_host_noalloc(np.zeros((5, mon.shape[1])), np.zeros((5, M.shape[1])),
                                     np.zeros((5, com.shape[1])), RHO, False, "fp64")
        assert e.value.code == -1 and "at most" in str(e.value)
    finally:
        ctx.close()
