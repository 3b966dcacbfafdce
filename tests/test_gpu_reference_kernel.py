"""The reference's own CUDA interaction kernels (built in place by
oracle/build_ref_gpu.sh with --fmad=false; test infrastructure, never part of
the library) against the oracle on the same staged SoA buffers: the
multipole kernel (RHO and d(rho)/dt, with leaf and empty neighbours) and the
P2P kernel. These kernels sum per stencil-column block and then add the 121
(M2L) or 11 (P2P) block partials in block order, a different summation order
from the reference's CPU sweep the oracle restates, so they agree to rounding
(1e-12 per component relative to its largest magnitude), not bit for bit. This
pins the comparator that tests/reference_gpu_timing.py times beside the
library's kernels."""
from __future__ import annotations

import numpy as np
import pytest

from octotiger_b200 import synthetic as syn
from octotiger_b200.layout import COMPONENT_LENGTH_UNPADDED, NCELL

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def refgpu():
    from oracle.pyoracle import REF_GPU_LIB, RefGpu
    if not REF_GPU_LIB.exists():
        pytest.skip("reference GPU build (oracle/_ref/libotfmm_ref_gpu.so) not present")
    return RefGpu(0.5)


def _cells(a, ncomp):
    return np.asarray(a).reshape(ncomp, -1)[:, :NCELL]


def _close(got, ref, tol=1e-12):
    scale = np.abs(ref).max(axis=1)
    assert (np.abs(got - ref).max(axis=1) <= tol * scale).all(), np.abs(got - ref).max(axis=1) / scale


@pytest.mark.parametrize("rho", [True, False])
@pytest.mark.parametrize("case", ["refined", "mixed"])
def test_reference_m2l_kernel_matches_oracle(refgpu, oracle, rho, case):
    import torch
    b = (syn.single_subgrid(seed=91) if case == "refined"
         else syn.single_subgrid(seed=92, leaf_dirs=(0, 6, 13, 19), empty_dirs=(2, 24)))
    mon, M, com = oracle.stage_m2l(b.pool, b.items[0])
    Lo, Lco = oracle.m2l_soa(0.5, mon, M, com, rho=rho, root=False)
    d = torch.device("cuda", 0)
    tm, tM, tc = (torch.from_numpy(x).to(d) for x in (mon, M, com))
    scratch = torch.zeros(refgpu.m2l_scratch(), dtype=torch.float64, device=d)
    L = torch.zeros(20 * COMPONENT_LENGTH_UNPADDED, dtype=torch.float64, device=d)
    Lc = torch.zeros(3 * COMPONENT_LENGTH_UNPADDED, dtype=torch.float64, device=d)
    refgpu.m2l(tm, tc, tM, scratch, L, Lc, rho=rho)
    torch.cuda.synchronize()
    _close(_cells(L.cpu().numpy(), 20), _cells(Lo, 20))
    if rho:
        _close(_cells(Lc.cpu().numpy(), 3), _cells(Lco, 3))


def test_reference_p2p_kernel_matches_oracle(refgpu, oracle):
    import torch
    b = syn.single_subgrid(seed=93, leaf_centre=True, leaf_dirs=tuple(range(0, 26, 2)), empty_dirs=(5,))
    mon = oracle.stage_p2p(b.pool, b.items[0])
    dx = float(b.items[0]["dx"])
    L4o = oracle.p2p_soa(0.5, mon, dx)
    d = torch.device("cuda", 0)
    scratch = torch.zeros(refgpu.p2p_scratch(), dtype=torch.float64, device=d)
    L4 = torch.zeros(4 * COMPONENT_LENGTH_UNPADDED, dtype=torch.float64, device=d)
    refgpu.p2p(torch.from_numpy(mon).to(d), scratch, L4, dx)
    torch.cuda.synchronize()
    _close(_cells(L4.cpu().numpy(), 4), _cells(L4o, 4))
