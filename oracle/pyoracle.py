"""TEST INFRASTRUCTURE ONLY — ctypes bindings of the oracle.

``Oracle`` wraps oracle/liboracle.so (the CPU restatement, always built by
``__graft_entry__.build()``). ``RefMath`` wraps oracle/_ref/libotfmm_ref_*.so,
the reference's own kernel arithmetic compiled by oracle/build_ref.sh, present
only where the reference tree was available at build time. Only tests/,
``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg use this module,
and only as the checker.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

from octotiger_b200.layout import (COMPONENT_LENGTH, COMPONENT_LENGTH_UNPADDED, ENTRIES,
                                   FULL_STENCIL_SIZE, NCELL, WORK_ITEM_DTYPE, SubgridPool)

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "liboracle.so"
REF_DIR = HERE / "_ref"

_dp = ctypes.POINTER(ctypes.c_double)
_u8p = ctypes.POINTER(ctypes.c_uint8)
_ip = ctypes.POINTER(ctypes.c_int)
_llp = ctypes.POINTER(ctypes.c_longlong)


def _ptr(a: np.ndarray, t=_dp):
    return a.ctypes.data_as(t)


def _check(rc: int, what: str) -> None:
    if rc < 0:
        raise RuntimeError(f"{what} failed with status {rc}")


class _Common:
    lib: ctypes.CDLL

    @staticmethod
    def _pool_args(pool: SubgridPool):
        pool.validate()
        return (_ptr(pool.M), _ptr(pool.com), _ptr(pool.mon), _ptr(pool.is_leaf, _u8p), ctypes.c_int(pool.n))

    # ------------------------------------------------------------ tree passes
    _up = "oracle_upward"
    _down = "oracle_downward"
    _shift = "oracle_shift"

    def shift(self, A: np.ndarray, X: np.ndarray, down: bool) -> np.ndarray:
        """taylor<4> shift of 20 moments / expansion coefficients by X."""
        A = np.ascontiguousarray(A, dtype=np.float64)
        X = np.ascontiguousarray(X, dtype=np.float64)
        B = np.zeros(20)
        getattr(self.lib, self._shift)(_ptr(A), _ptr(X), _ptr(B), int(down))
        return B

    def upward(self, pool: SubgridPool, nodes: np.ndarray, level_start: np.ndarray, rho: bool = True,
               com1: np.ndarray | None = None):
        """Upward pass on copies of the pool: returns (M, com, com1)."""
        M = pool.M.copy()
        com = pool.com.copy()
        com1 = np.zeros((pool.n, 3, 64)) if com1 is None else com1.copy()
        nodes = np.ascontiguousarray(nodes)
        ls = np.ascontiguousarray(level_start, dtype=np.int32)
        rc = getattr(self.lib, self._up)(_ptr(M), _ptr(com), _ptr(pool.mon), _ptr(pool.is_leaf, _u8p),
                                         _ptr(com1), ctypes.c_int(pool.n), nodes.ctypes.data_as(ctypes.c_void_p),
                                         _ptr(ls, _ip), ctypes.c_int(len(ls) - 1), int(rho))
        _check(rc, self._up)
        return M, com, com1

    def downward(self, com, is_leaf, com1, nodes, level_start, L, Lc, gconst: float = 1.0,
                 correct_am: bool = True, rho: bool = True):
        """Downward pass on copies of L, L_c: returns (L, L_c, G)."""
        L = np.ascontiguousarray(L, dtype=np.float64).copy()
        Lc = np.ascontiguousarray(Lc, dtype=np.float64).copy()
        G = np.zeros((L.shape[0], 4, NCELL))
        com = np.ascontiguousarray(com, dtype=np.float64)
        com1 = np.ascontiguousarray(com1, dtype=np.float64)
        is_leaf = np.ascontiguousarray(is_leaf, dtype=np.uint8)
        nodes = np.ascontiguousarray(nodes)
        ls = np.ascontiguousarray(level_start, dtype=np.int32)
        rc = getattr(self.lib, self._down)(_ptr(com), _ptr(is_leaf, _u8p), _ptr(com1), ctypes.c_int(L.shape[0]),
                                           nodes.ctypes.data_as(ctypes.c_void_p), _ptr(ls, _ip),
                                           ctypes.c_int(len(ls) - 1), _ptr(L), _ptr(Lc), _ptr(G),
                                           ctypes.c_double(gconst), int(correct_am), int(rho))
        _check(rc, self._down)
        return L, Lc, G



class Oracle(_Common):
    def __init__(self, path: Path = ORACLE_SO):
        if not Path(path).exists():
            raise FileNotFoundError(f"oracle library missing: {path} (run make -C oracle)")
        self.lib = ctypes.CDLL(str(path))

    def stencil(self, theta: float) -> dict:
        mm = np.zeros(FULL_STENCIL_SIZE, np.uint8)
        ph = np.zeros(FULL_STENCIL_SIZE, np.uint8)
        pm = np.zeros(FULL_STENCIL_SIZE, np.uint8)
        four = np.zeros((FULL_STENCIL_SIZE, 4))
        counts = np.zeros(3, np.int32)
        rc = self.lib.oracle_build_stencil(ctypes.c_double(theta), _ptr(mm, _u8p), _ptr(ph, _u8p), _ptr(pm, _u8p),
                                           _ptr(four), _ptr(counts, _ip))
        _check(rc, "oracle_build_stencil")
        return dict(mpole_mask=mm, mpole_phase=ph, p2p_mask=pm, four=four, n_mpole=int(counts[0]),
                    n_phase_one=int(counts[1]), n_p2p=int(counts[2]))

    def m2l_soa(self, theta, mon, M, com, rho=True, root=False):
        L = np.zeros(20 * COMPONENT_LENGTH_UNPADDED)
        Lc = np.zeros(3 * COMPONENT_LENGTH_UNPADDED)
        rc = self.lib.oracle_m2l_soa(ctypes.c_double(theta), _ptr(mon), _ptr(M), _ptr(com), _ptr(L), _ptr(Lc),
                                     int(rho), int(root))
        _check(rc, "oracle_m2l_soa")
        return L, Lc

    def p2p_soa(self, theta, mon, dx):
        L4 = np.zeros(4 * COMPONENT_LENGTH_UNPADDED)
        _check(self.lib.oracle_p2p_soa(ctypes.c_double(theta), _ptr(mon), ctypes.c_double(dx), _ptr(L4)),
               "oracle_p2p_soa")
        return L4

    def p2m_dir(self, theta, d, nM, ncom, stride, icom, L4, Lc, rho=True, reset=True):
        _check(self.lib.oracle_p2m_dir(ctypes.c_double(theta), int(d), _ptr(nM), _ptr(ncom), int(stride),
                                       _ptr(icom), _ptr(L4), _ptr(Lc), int(rho), int(reset)), "oracle_p2m_dir")

    def stage_m2l(self, pool: SubgridPool, item):
        mon = np.zeros(ENTRIES)
        M = np.zeros(20 * COMPONENT_LENGTH)
        com = np.zeros(3 * COMPONENT_LENGTH)
        it = np.ascontiguousarray(np.asarray(item, dtype=WORK_ITEM_DTYPE).reshape(1))
        _check(self.lib.oracle_stage_m2l(*self._pool_args(pool), it.ctypes.data_as(ctypes.c_void_p), _ptr(mon),
                                         _ptr(M), _ptr(com)), "oracle_stage_m2l")
        return mon, M, com

    def stage_p2p(self, pool: SubgridPool, item):
        mon = np.zeros(ENTRIES)
        it = np.ascontiguousarray(np.asarray(item, dtype=WORK_ITEM_DTYPE).reshape(1))
        _check(self.lib.oracle_stage_p2p(*self._pool_args(pool), it.ctypes.data_as(ctypes.c_void_p), _ptr(mon)),
               "oracle_stage_p2p")
        return mon

    def stage_p2m(self, pool: SubgridPool, nb: int, d: int):
        nM = np.zeros(20 * 419)
        ncom = np.zeros(3 * 419)
        stride = self.lib.oracle_stage_p2m(*self._pool_args(pool), int(nb), int(d), _ptr(nM), _ptr(ncom))
        _check(stride, "oracle_stage_p2m")
        return nM, ncom, int(stride)

    def batch(self, theta, pool: SubgridPool, items: np.ndarray, rho=True, nthreads=None):
        L = np.zeros((pool.n, 20, NCELL))
        Lc = np.zeros((pool.n, 3, NCELL))
        nthreads = nthreads or os.cpu_count() or 1
        rc = self.lib.oracle_batch(ctypes.c_double(theta), *self._pool_args(pool),
                                   items.ctypes.data_as(ctypes.c_void_p), ctypes.c_int(len(items)), int(rho),
                                   _ptr(L), _ptr(Lc), int(nthreads))
        _check(rc, "oracle_batch")
        return L, Lc

    def count_pairs(self, theta, pool: SubgridPool, items: np.ndarray):
        """Total evaluated pairs and the split [M2L, root M2L, P2P, P2M]."""
        per = np.zeros(4, np.int64)
        self.lib.oracle_count_pairs.restype = ctypes.c_longlong
        tot = self.lib.oracle_count_pairs(ctypes.c_double(theta), _ptr(pool.is_leaf, _u8p), ctypes.c_int(pool.n),
                                          items.ctypes.data_as(ctypes.c_void_p), ctypes.c_int(len(items)),
                                          _ptr(per, _llp))
        _check(tot, "oracle_count_pairs")
        return int(tot), per


def host_has_avx512() -> bool:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("flags"):
                    return " avx512f" in line
    except OSError:
        pass
    return False


def ref_library_path() -> Path | None:
    """The reference-math build that runs on this host, or None."""
    cands = ["avx512", "avx2"] if host_has_avx512() else ["avx2"]
    for c in cands:
        p = REF_DIR / f"libotfmm_ref_{c}.so"
        if p.exists():
            return p
    return None


class RefMath(_Common):
    """The reference's own kernel arithmetic (SIMD lanes along z; the tree
    passes through its taylor<4> shift operators)."""

    _up = "ref_upward"
    _down = "ref_downward"
    _shift = "ref_shift"

    def __init__(self, path: Path | None = None):
        path = path or ref_library_path()
        if path is None or not Path(path).exists():
            raise FileNotFoundError("reference-math build missing (run oracle/build_ref.sh)")
        self.path = Path(path)
        self.lib = ctypes.CDLL(str(path))

    def simd_width(self, simd=True) -> int:
        return int(self.lib.ref_simd_width(int(simd)))

    def stencil(self, theta: float) -> dict:
        mm = np.zeros(FULL_STENCIL_SIZE, np.uint8)
        ph = np.zeros(FULL_STENCIL_SIZE, np.uint8)
        pm = np.zeros(FULL_STENCIL_SIZE, np.uint8)
        four = np.zeros((FULL_STENCIL_SIZE, 4))
        _check(self.lib.ref_build_stencil(ctypes.c_double(theta), _ptr(mm, _u8p), _ptr(ph, _u8p), _ptr(pm, _u8p),
                                          _ptr(four)), "ref_build_stencil")
        return dict(mpole_mask=mm, mpole_phase=ph, p2p_mask=pm, four=four)

    def m2l_soa(self, theta, mon, M, com, rho=True, root=False, simd=True):
        L = np.zeros(20 * COMPONENT_LENGTH_UNPADDED)
        Lc = np.zeros(3 * COMPONENT_LENGTH_UNPADDED)
        _check(self.lib.ref_m2l_soa(int(simd), ctypes.c_double(theta), _ptr(mon), _ptr(M), _ptr(com), _ptr(L),
                                    _ptr(Lc), int(rho), int(root)), "ref_m2l_soa")
        return L, Lc

    def p2p_soa(self, theta, mon, dx, simd=True):
        L4 = np.zeros(4 * COMPONENT_LENGTH_UNPADDED)
        _check(self.lib.ref_p2p_soa(int(simd), ctypes.c_double(theta), _ptr(mon), ctypes.c_double(dx), _ptr(L4)),
               "ref_p2p_soa")
        return L4

    def p2m_dir(self, theta, d, nM, ncom, stride, icom, L4, Lc, rho=True, reset=True, simd=True):
        _check(self.lib.ref_p2m_dir(int(simd), ctypes.c_double(theta), int(d), _ptr(nM), _ptr(ncom), int(stride),
                                    _ptr(icom), _ptr(L4), _ptr(Lc), int(rho), int(reset)), "ref_p2m_dir")

    def batch(self, theta, pool: SubgridPool, items: np.ndarray, rho=True, nthreads=None, simd=True):
        L = np.zeros((pool.n, 20, NCELL))
        Lc = np.zeros((pool.n, 3, NCELL))
        nthreads = nthreads or os.cpu_count() or 1
        rc = self.lib.ref_batch(int(simd), ctypes.c_double(theta), *self._pool_args(pool),
                                items.ctypes.data_as(ctypes.c_void_p), ctypes.c_int(len(items)), int(rho), _ptr(L),
                                _ptr(Lc), int(nthreads))
        _check(rc, "ref_batch")
        return L, Lc


REF_GPU_LIB = REF_DIR / "libotfmm_ref_gpu.so"


class RefGpu:
    """The reference's own CUDA interaction kernels (oracle/build_ref_gpu.sh),
    run on device buffers in the reference's SoA layout: a comparator for the
    GPU tests and the timing script, never part of the library."""

    def __init__(self, theta: float = 0.5, path: Path = REF_GPU_LIB):
        if not Path(path).exists():
            raise FileNotFoundError("reference GPU build missing (run oracle/build_ref_gpu.sh)")
        self.lib = ctypes.CDLL(str(path))
        vp, dp, i = ctypes.c_void_p, ctypes.c_double, ctypes.c_int
        self.lib.refgpu_init.argtypes = [dp]
        self.lib.refgpu_m2l.argtypes = [vp, vp, vp, vp, vp, vp, dp, i, vp]
        self.lib.refgpu_p2p.argtypes = [vp, vp, vp, dp, dp, vp]
        self.lib.refgpu_m2l_scratch_doubles.restype = ctypes.c_size_t
        self.lib.refgpu_p2p_scratch_doubles.restype = ctypes.c_size_t
        self.theta = float(theta)
        _check(self.lib.refgpu_init(self.theta), "refgpu_init")

    def m2l_scratch(self) -> int:
        return int(self.lib.refgpu_m2l_scratch_doubles())

    def p2p_scratch(self) -> int:
        return int(self.lib.refgpu_p2p_scratch_doubles())

    def m2l(self, mon, com, M, scratch, L, Lc, rho=True, stream=0):
        """Device pointers (ints) or torch tensors; asynchronous on `stream`."""
        p = [t if isinstance(t, int) else t.data_ptr() for t in (mon, com, M, scratch, L, Lc)]
        _check(self.lib.refgpu_m2l(*p, self.theta, int(rho), stream), "refgpu_m2l")

    def p2p(self, mon, scratch, L4, dx, stream=0):
        p = [t if isinstance(t, int) else t.data_ptr() for t in (mon, scratch, L4)]
        _check(self.lib.refgpu_p2p(*p, self.theta, float(dx), stream), "refgpu_p2p")
