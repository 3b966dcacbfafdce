"""Host binding of libotfmm.so (the C ABI in include/otfmm.h).

Device memory and streams come from PyTorch; the kernels are the library's.
There is no CPU fallback: without the built library or a CUDA device every
entry point raises.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from pathlib import Path

import numpy as np

from .layout import (COMPONENT_LENGTH, COMPONENT_LENGTH_UNPADDED, ENTRIES, NCELL, RHO, WORK_ITEM_DTYPE,
                     SubgridPool, validate_work_list)

LIB_PATH = Path(__file__).resolve().parent / "libotfmm.so"

OTFMM_OK = 0
ERRORS = {-1: "invalid argument", -2: "theta below minimum", -3: "CUDA error", -4: "device-side work item error",
          -5: "unsupported"}
FP64_EXACT, FP64, FP32_SPLIT = 0, 1, 2
PRECISIONS = {"fp64_exact": FP64_EXACT, "fp64": FP64, "fp32_split": FP32_SPLIT}

EXPORTED = ["otfmm_create", "otfmm_destroy", "otfmm_stencil_info", "otfmm_m2l_soa", "otfmm_m2l_soa_host",
            "otfmm_p2p_soa", "otfmm_p2m_soa", "otfmm_batch", "otfmm_batch_status", "otfmm_count_pairs",
            "otfmm_m2l_soa_host_noalloc", "otfmm_stage_soa", "otfmm_stage_p2m_soa", "otfmm_get_tuning",
            "otfmm_set_tuning", "otfmm_autotune", "otfmm_batch_profile", "otfmm_batch_host", "otfmm_upward",
            "otfmm_downward", "otfmm_plan_create", "otfmm_plan_launch", "otfmm_plan_status",
            "otfmm_plan_destroy", "otfmm_last_error",
            "otfmm_build_info", "otfmm_measure_fma_peaks"]

_lib = None

SPLIT_WARP_SPECIALISED, SPLIT_SINGLE_ROLE, SPLIT_WARP_SPECIALISED_PACKED, SPLIT_FUSED = 0, 1, 2, 3
SPLIT_FORMS = {0: "warp_specialised", 1: "single_role", 2: "warp_specialised_packed", 3: "fused"}
P2P_FORMS = {0: "box", 1: "stencil"}
P2M_FORMS = {0: "coarse", 1: "lanes", 2: "octant"}


class Tuning(ctypes.Structure):
    """otfmm_tuning: the kernel variants of the batched solve."""
    _fields_ = [("split_m2l_form", ctypes.c_int32), ("split_m2l_chunk", ctypes.c_int32),
                ("split_p2p_chunk", ctypes.c_int32), ("p2m_lanes", ctypes.c_int32), ("p2p_form", ctypes.c_int32),
                ("p2m_form", ctypes.c_int32)]

    def as_dict(self) -> dict:
        return {"split_m2l_form": SPLIT_FORMS.get(self.split_m2l_form, str(self.split_m2l_form)),
                "split_m2l_chunk": self.split_m2l_chunk, "split_p2p_chunk": self.split_p2p_chunk,
                "p2m_lanes": self.p2m_lanes, "p2p_form": P2P_FORMS.get(self.p2p_form, str(self.p2p_form)),
                "p2m_form": P2M_FORMS.get(self.p2m_form, str(self.p2m_form))}


class OtfmmError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"otfmm error {code} ({ERRORS.get(code, '?')}): {msg}")
        self.code = code


def load_library(path: Path = LIB_PATH) -> ctypes.CDLL:
    """Loads libotfmm.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not Path(path).exists():
            raise FileNotFoundError(f"{path} not built: run `python -m octotiger_b200.build`")
        lib = ctypes.CDLL(str(path))
        vp, dp, i = ctypes.c_void_p, ctypes.c_double, ctypes.c_int
        lib.otfmm_create.argtypes = [i, dp, ctypes.POINTER(vp)]
        lib.otfmm_destroy.argtypes = [vp]
        lib.otfmm_stencil_info.argtypes = [vp, vp, vp, vp, vp]
        lib.otfmm_m2l_soa.argtypes = [vp, vp, vp, vp, vp, vp, i, i, i, vp]
        lib.otfmm_m2l_soa_host.argtypes = [vp, vp, vp, vp, vp, vp, i, i, i]
        lib.otfmm_m2l_soa_host_noalloc.argtypes = [vp, ctypes.c_int32, vp, vp, vp, vp, vp, i, i, i, vp]
        lib.otfmm_p2p_soa.argtypes = [vp, vp, dp, vp, i, vp]
        lib.otfmm_p2m_soa.argtypes = [vp, i, vp, vp, vp, vp, vp, i, i, i, vp]
        lib.otfmm_batch.argtypes = [vp, vp, vp, vp, vp, ctypes.c_int32, vp, ctypes.c_int32, vp, vp, i, i, vp]
        lib.otfmm_batch_status.argtypes = [vp, vp]
        lib.otfmm_get_tuning.argtypes = [vp, ctypes.POINTER(Tuning)]
        lib.otfmm_set_tuning.argtypes = [vp, ctypes.POINTER(Tuning)]
        lib.otfmm_autotune.argtypes = [vp, vp, vp, vp, vp, ctypes.c_int32, vp, ctypes.c_int32, vp, vp, i, i, i,
                                       ctypes.POINTER(Tuning), vp]
        lib.otfmm_plan_create.argtypes = [vp, vp, vp, vp, vp, ctypes.c_int32, vp, ctypes.c_int32, vp, vp, i, i,
                                          ctypes.POINTER(vp)]
        lib.otfmm_plan_create_host.argtypes = [vp, vp, vp, vp, vp, ctypes.c_int32, vp, ctypes.c_int32, vp, vp, i,
                                               i, ctypes.POINTER(vp)]
        lib.otfmm_plan_launch.argtypes = [vp, vp]
        lib.otfmm_upward.argtypes = [vp, vp, vp, vp, vp, vp, ctypes.c_int32, vp, vp, ctypes.c_int32, i, vp]
        lib.otfmm_downward.argtypes = [vp, vp, vp, vp, ctypes.c_int32, vp, vp, ctypes.c_int32, vp, vp, vp, dp, i, i,
                                       vp]
        lib.otfmm_batch_host.argtypes = [vp, vp, vp, vp, vp, ctypes.c_int32, vp, ctypes.c_int32, vp, vp, i, i, vp]
        lib.otfmm_batch_profile.argtypes = [vp, vp, vp, vp, vp, ctypes.c_int32, vp, ctypes.c_int32, vp, vp, i, i,
                                            ctypes.POINTER(ctypes.c_float), vp]
        lib.otfmm_plan_status.argtypes = [vp, vp]
        lib.otfmm_plan_destroy.argtypes = [vp]
        lib.otfmm_stage_soa.argtypes = [vp, vp, vp, vp, vp, ctypes.c_int32, vp, vp, vp, vp, vp]
        lib.otfmm_stage_p2m_soa.argtypes = [vp, vp, vp, ctypes.c_int32, ctypes.c_int32, i, vp, vp,
                                            ctypes.POINTER(ctypes.c_int32), vp]
        lib.otfmm_count_pairs.argtypes = [vp, vp, ctypes.c_int32, vp, ctypes.c_int32, vp]
        lib.otfmm_count_pairs.restype = ctypes.c_longlong
        lib.otfmm_last_error.restype = ctypes.c_char_p
        lib.otfmm_build_info.restype = ctypes.c_char_p
        lib.otfmm_measure_fma_peaks.argtypes = [i, ctypes.POINTER(dp), ctypes.POINTER(dp)]
        _lib = lib
    return _lib


def _check(rc: int) -> None:
    if rc != OTFMM_OK:
        raise OtfmmError(rc, load_library().otfmm_last_error().decode())


def _require_cuda():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("octotiger_b200 kernels need a CUDA device; there is no CPU fallback")
    return torch


def _ptr(t) -> ctypes.c_void_p:
    return ctypes.c_void_p(t.data_ptr()) if t is not None else ctypes.c_void_p(0)


def _stream(stream) -> ctypes.c_void_p:
    if stream is None:
        import torch
        stream = torch.cuda.current_stream()
    return ctypes.c_void_p(stream.cuda_stream)


def precision_code(precision) -> int:
    return PRECISIONS[precision] if isinstance(precision, str) else int(precision)


class Context:
    """A library context: device, opening angle and its stencil tables."""

    def __init__(self, device: int = 0, theta: float = 0.5):
        _require_cuda()
        lib = load_library()
        h = ctypes.c_void_p()
        _check(lib.otfmm_create(int(device), float(theta), ctypes.byref(h)))
        self.handle = h
        self.device = device
        self.theta = theta

    def close(self) -> None:
        if getattr(self, "handle", None):
            load_library().otfmm_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def stencil_info(self) -> dict:
        counts = np.zeros(3, np.int32)
        mm = np.zeros(1331, np.uint8)
        ph = np.zeros(1331, np.uint8)
        pm = np.zeros(1331, np.uint8)
        _check(load_library().otfmm_stencil_info(self.handle, counts.ctypes.data, mm.ctypes.data, ph.ctypes.data,
                                                 pm.ctypes.data))
        return dict(n_mpole=int(counts[0]), n_phase_one=int(counts[1]), n_p2p=int(counts[2]), mpole_mask=mm,
                    mpole_phase=ph, p2p_mask=pm)

    # ---------------------------------------------------------------- per subgrid (reference SoA layout)
    def m2l_soa(self, mon, M, com, L, Lc, gsolve_type=RHO, use_root_stencil=False, precision=FP64, stream=None):
        """Device tensors in the reference's SoA layout (see include/otfmm.h)."""
        _check(load_library().otfmm_m2l_soa(self.handle, _ptr(mon), _ptr(M), _ptr(com), _ptr(L), _ptr(Lc),
                                            int(gsolve_type), int(bool(use_root_stencil)),
                                            precision_code(precision), _stream(stream)))

    def m2l_soa_host(self, mon: np.ndarray, M: np.ndarray, com: np.ndarray, gsolve_type=RHO,
                     use_root_stencil=False, precision=FP64):
        """Host buffers in, host buffers out (the reference's launch_interface)."""
        L = np.zeros(20 * COMPONENT_LENGTH_UNPADDED)
        Lc = np.zeros(3 * COMPONENT_LENGTH_UNPADDED)
        for a, n in ((mon, ENTRIES), (M, 20 * COMPONENT_LENGTH), (com, 3 * COMPONENT_LENGTH)):
            if a is not None and (a.dtype != np.float64 or a.size < n or not a.flags.c_contiguous):
                raise ValueError("SoA buffers must be contiguous float64 of the reference sizes")
        _check(load_library().otfmm_m2l_soa_host(
            self.handle, None if mon is None else mon.ctypes.data, M.ctypes.data, com.ctypes.data, L.ctypes.data,
            Lc.ctypes.data, int(gsolve_type), int(bool(use_root_stencil)), precision_code(precision)))
        return L, Lc

    def m2l_soa_host_noalloc(self, mon, M, com, gsolve_type=RHO, use_root_stencil=False, precision=FP64):
        """Host-buffer multipole call for 1..4 subgrids that allocates no device
        memory (its staging is a static device array). Inputs are stacked per
        subgrid: mon [n, 5832] (None for the root stencil), M [n, 20*5851],
        com [n, 3*5851]; returns L [n, 20*531], L_c [n, 3*531]."""
        M = np.ascontiguousarray(M, dtype=np.float64).reshape(-1, 20 * COMPONENT_LENGTH)
        com = np.ascontiguousarray(com, dtype=np.float64).reshape(-1, 3 * COMPONENT_LENGTH)
        n = M.shape[0]
        if mon is not None:
            mon = np.ascontiguousarray(mon, dtype=np.float64).reshape(-1, ENTRIES)
            if mon.shape[0] != n:
                raise ValueError("mon and M disagree on the number of subgrids")
        if com.shape[0] != n:
            raise ValueError("com and M disagree on the number of subgrids")
        L = np.zeros((n, 20 * COMPONENT_LENGTH_UNPADDED))
        Lc = np.zeros((n, 3 * COMPONENT_LENGTH_UNPADDED))
        _check(load_library().otfmm_m2l_soa_host_noalloc(
            self.handle, ctypes.c_int32(n), None if mon is None else mon.ctypes.data, M.ctypes.data,
            com.ctypes.data, L.ctypes.data, Lc.ctypes.data, int(gsolve_type), int(bool(use_root_stencil)),
            precision_code(precision), None))
        return L, Lc

    def p2p_soa(self, mon, dx, L4, precision=FP64, stream=None):
        _check(load_library().otfmm_p2p_soa(self.handle, _ptr(mon), float(dx), _ptr(L4), precision_code(precision),
                                            _stream(stream)))

    def p2m_soa(self, d, nM, ncom, icom, L4, Lc, gsolve_type=RHO, reset_lc=True, precision=FP64, stream=None):
        _check(load_library().otfmm_p2m_soa(self.handle, int(d), _ptr(nM), _ptr(ncom), _ptr(icom), _ptr(L4),
                                            _ptr(Lc), int(gsolve_type), int(bool(reset_lc)),
                                            precision_code(precision), _stream(stream)))

    def stage_soa(self, dev: "DevicePool", item: np.ndarray, mon, M=None, com=None, stream=None) -> None:
        """Device-side update_input of one work item (numpy record) from a
        resident pool into the reference's SoA buffers (device tensors)."""
        it = np.ascontiguousarray(np.asarray(item).reshape(1))
        _check(load_library().otfmm_stage_soa(self.handle, _ptr(dev.M), _ptr(dev.com), _ptr(dev.mon),
                                              _ptr(dev.is_leaf), ctypes.c_int32(dev.n), it.ctypes.data, _ptr(mon),
                                              _ptr(M), _ptr(com), _stream(stream)))

    def stage_p2m_soa(self, dev: "DevicePool", neighbor: int, d: int, nM, ncom, stream=None) -> int:
        """Refined neighbour slab for otfmm_p2m_soa; returns its component stride."""
        stride = ctypes.c_int32()
        _check(load_library().otfmm_stage_p2m_soa(self.handle, _ptr(dev.M), _ptr(dev.com), ctypes.c_int32(dev.n),
                                                  ctypes.c_int32(int(neighbor)), int(d), _ptr(nM), _ptr(ncom),
                                                  ctypes.byref(stride), _stream(stream)))
        return stride.value

    # ---------------------------------------------------------------- batched
    def batch(self, dev: "DevicePool", items_dev, n_items: int, L, Lc, gsolve_type=RHO, precision=FP64,
              stream=None):
        _check(load_library().otfmm_batch(self.handle, _ptr(dev.M), _ptr(dev.com), _ptr(dev.mon), _ptr(dev.is_leaf),
                                          ctypes.c_int32(dev.n), _ptr(items_dev), ctypes.c_int32(n_items), _ptr(L),
                                          _ptr(Lc), int(gsolve_type), precision_code(precision), _stream(stream)))

    def batch_host(self, M, com, mon, is_leaf, n_subgrids: int, items, n_items: int, L, Lc, gsolve_type=RHO,
                   precision=FP64, stream=None) -> None:
        """Batched solve from host buffers (numpy arrays or pinned CPU torch
        tensors): pipelined uploads, kernels and downloads; L / Lc are
        complete once `stream` has finished. Calls of one context on
        different streams must not overlap (they share its device copies)."""
        hp = _host_ptr
        _check(load_library().otfmm_batch_host(self.handle, hp(M), hp(com), hp(mon), hp(is_leaf),
                                               ctypes.c_int32(n_subgrids), hp(items), ctypes.c_int32(n_items),
                                               hp(L), hp(Lc), int(gsolve_type), precision_code(precision),
                                               _stream(stream)))

    def plan_host(self, M, com, mon, is_leaf, n_subgrids: int, items, n_items: int, L, Lc, gsolve_type=RHO,
                  precision=FP64) -> "Plan":
        """batch_host captured once for these pinned host buffers (see
        otfmm_plan_create_host); launch() replays the whole host-buffer solve."""
        return Plan.from_host(self, M, com, mon, is_leaf, n_subgrids, items, n_items, L, Lc, gsolve_type, precision)

    def upward(self, dev: "DevicePool", com1, nodes_dev, level_start: np.ndarray, gsolve_type=RHO,
               stream=None) -> None:
        """M2M pass (see otfmm_upward): fills the refined nodes' M / com and com1."""
        ls = np.ascontiguousarray(level_start, dtype=np.int32)
        _check(load_library().otfmm_upward(self.handle, _ptr(dev.M), _ptr(dev.com), _ptr(dev.mon), _ptr(dev.is_leaf),
                                           _ptr(com1), ctypes.c_int32(dev.n), _ptr(nodes_dev), ls.ctypes.data,
                                           ctypes.c_int32(len(ls) - 1), int(gsolve_type), _stream(stream)))

    def downward(self, dev: "DevicePool", com1, nodes_dev, level_start: np.ndarray, L, Lc, G, gconst=1.0,
                 correct_am_grav=True, gsolve_type=RHO, stream=None) -> None:
        """L2L pass (see otfmm_downward): adds the parents' expansions to L / L_c, writes G of leaves."""
        ls = np.ascontiguousarray(level_start, dtype=np.int32)
        _check(load_library().otfmm_downward(self.handle, _ptr(dev.com), _ptr(dev.is_leaf), _ptr(com1),
                                             ctypes.c_int32(dev.n), _ptr(nodes_dev), ls.ctypes.data,
                                             ctypes.c_int32(len(ls) - 1), _ptr(L), _ptr(Lc), _ptr(G),
                                             float(gconst), int(bool(correct_am_grav)), int(gsolve_type),
                                             _stream(stream)))

    def batch_profile(self, dev: "DevicePool", items_dev, n_items: int, L, Lc, gsolve_type=RHO, precision=FP64,
                      stream=None) -> dict:
        """One batched solve with per-kernel device times (ms)."""
        ms = (ctypes.c_float * 4)()
        _check(load_library().otfmm_batch_profile(self.handle, _ptr(dev.M), _ptr(dev.com), _ptr(dev.mon),
                                                  _ptr(dev.is_leaf), ctypes.c_int32(dev.n), _ptr(items_dev),
                                                  ctypes.c_int32(n_items), _ptr(L), _ptr(Lc), int(gsolve_type),
                                                  precision_code(precision), ms, _stream(stream)))
        return {"classify": ms[0], "m2l": ms[1], "p2p": ms[2], "p2m": ms[3]}

    def get_tuning(self) -> Tuning:
        t = Tuning()
        _check(load_library().otfmm_get_tuning(self.handle, ctypes.byref(t)))
        return t

    def set_tuning(self, t: Tuning) -> None:
        _check(load_library().otfmm_set_tuning(self.handle, ctypes.byref(t)))

    def autotune(self, dev: "DevicePool", items_dev, n_items: int, L, Lc, gsolve_type=RHO, precision=FP64,
                 repeats: int = 3, stream=None) -> Tuning:
        """Times the kernel variants on this batch and keeps the fastest."""
        t = Tuning()
        _check(load_library().otfmm_autotune(self.handle, _ptr(dev.M), _ptr(dev.com), _ptr(dev.mon),
                                             _ptr(dev.is_leaf), ctypes.c_int32(dev.n), _ptr(items_dev),
                                             ctypes.c_int32(n_items), _ptr(L), _ptr(Lc), int(gsolve_type),
                                             precision_code(precision), int(repeats), ctypes.byref(t),
                                             _stream(stream)))
        return t

    def count_pairs(self, is_leaf: np.ndarray, items: np.ndarray) -> tuple[int, np.ndarray]:
        """Cell-interactions of a work list: total and [M2L, root, P2P, P2M]."""
        per = np.zeros(4, np.int64)
        items = np.ascontiguousarray(items)
        is_leaf = np.ascontiguousarray(is_leaf, dtype=np.uint8)
        tot = load_library().otfmm_count_pairs(self.handle, is_leaf.ctypes.data, ctypes.c_int32(len(is_leaf)),
                                               items.ctypes.data, ctypes.c_int32(len(items)), per.ctypes.data)
        if tot < 0:
            _check(int(tot))
        return int(tot), per

    def batch_status(self, stream=None) -> None:
        _check(load_library().otfmm_batch_status(self.handle, _stream(stream)))


@dataclass
class DevicePool:
    """A subgrid pool resident on the GPU (torch tensors)."""

    M: object
    com: object
    mon: object
    is_leaf: object
    n: int

    @classmethod
    def upload(cls, pool: SubgridPool, device: int = 0, non_blocking: bool = False) -> "DevicePool":
        torch = _require_cuda()
        pool.validate()
        dev = torch.device("cuda", device)
        t = {k: torch.from_numpy(getattr(pool, k)).to(dev, non_blocking=non_blocking)
             for k in ("M", "com", "mon", "is_leaf")}
        return cls(n=pool.n, **t)


def order_work_list(items: np.ndarray) -> np.ndarray:
    """Multipole (heaviest) items first: the block scheduler then fills the
    GPU with the long tiles and ends with the short leaf tiles."""
    key = np.where(items["kind"] == 2, 1, 0)
    return np.ascontiguousarray(items[np.argsort(key, kind="stable")])


def upload_work_list(items: np.ndarray, n_subgrids: int, device: int = 0):
    torch = _require_cuda()
    validate_work_list(items, n_subgrids)
    raw = np.ascontiguousarray(items).view(np.uint8).reshape(-1)
    return torch.from_numpy(raw.copy()).to(torch.device("cuda", device))


class BatchSolver:
    """Runs one gravity solve's work list on the GPU from a resident pool."""

    def __init__(self, ctx: Context, pool: SubgridPool, items: np.ndarray):
        torch = _require_cuda()
        self.ctx = ctx
        self.dev = DevicePool.upload(pool, ctx.device)
        self.items_host = order_work_list(items)
        self.items = upload_work_list(self.items_host, pool.n, ctx.device)
        self.n_items = len(items)
        d = torch.device("cuda", ctx.device)
        self.L = torch.zeros((pool.n, 20, NCELL), dtype=torch.float64, device=d)
        self.Lc = torch.zeros((pool.n, 3, NCELL), dtype=torch.float64, device=d)

    @classmethod
    def from_device(cls, ctx: Context, dev: DevicePool, items: np.ndarray) -> "BatchSolver":
        """A solve over records already resident on the context's device (for
        example a rank's shard after its halo exchange), with no host copy."""
        torch = _require_cuda()
        n = int(dev.n)
        if tuple(dev.M.shape) != (n, 20, NCELL) or tuple(dev.com.shape) != (n, 3, NCELL) or \
                tuple(dev.mon.shape) != (n, NCELL) or tuple(dev.is_leaf.shape) != (n,):
            raise ValueError("device pool arrays have inconsistent shapes")
        if dev.M.dtype != torch.float64 or dev.is_leaf.dtype != torch.uint8:
            raise ValueError("device pool: float64 records and uint8 leaf flags expected")
        self = cls.__new__(cls)
        self.ctx = ctx
        self.dev = DevicePool(M=dev.M.contiguous(), com=dev.com.contiguous(), mon=dev.mon.contiguous(),
                              is_leaf=dev.is_leaf.contiguous(), n=n)
        self.items_host = order_work_list(items)
        self.items = upload_work_list(self.items_host, n, ctx.device)
        self.n_items = len(items)
        d = torch.device("cuda", ctx.device)
        self.L = torch.zeros((n, 20, NCELL), dtype=torch.float64, device=d)
        self.Lc = torch.zeros((n, 3, NCELL), dtype=torch.float64, device=d)
        return self

    def run(self, gsolve_type=RHO, precision=FP64, stream=None) -> None:
        self.ctx.batch(self.dev, self.items, self.n_items, self.L, self.Lc, gsolve_type, precision, stream)

    def results(self):
        self.ctx.batch_status()
        return self.L.cpu().numpy(), self.Lc.cpu().numpy()

    def profile(self, gsolve_type=RHO, precision=FP64) -> dict:
        return self.ctx.batch_profile(self.dev, self.items, self.n_items, self.L, self.Lc, gsolve_type, precision)

    def autotune(self, gsolve_type=RHO, precision=FP64, repeats: int = 3) -> Tuning:
        return self.ctx.autotune(self.dev, self.items, self.n_items, self.L, self.Lc, gsolve_type, precision, repeats)

    def plan(self, gsolve_type=RHO, precision=FP64) -> "Plan":
        """This solve captured into a CUDA graph (see otfmm_plan_create)."""
        return Plan(self.ctx, self.dev, self.items, self.n_items, self.L, self.Lc, gsolve_type, precision)


class GravitySolver:
    """A whole gravity solve on the device (node_server::solve_gravity's
    order): the upward pass (M2M) fills the refined nodes' multipoles from the
    leaves' masses, the batched interaction kernels fill L / L_c, the downward
    pass (L2L) adds the parents' expansions and writes the leaves' potential
    and acceleration G[n][4][512]."""

    def __init__(self, ctx: Context, pool: SubgridPool, items: np.ndarray, nodes: np.ndarray,
                 level_start: np.ndarray, gconst: float = 1.0, correct_am_grav: bool = True):
        torch = _require_cuda()
        self.batch = BatchSolver(ctx, pool, items)
        self.ctx = ctx
        d = torch.device("cuda", ctx.device)
        raw = np.ascontiguousarray(nodes).view(np.uint8).reshape(-1)
        self.nodes = torch.from_numpy(raw.copy()).to(d)
        self.level_start = np.ascontiguousarray(level_start, dtype=np.int32)
        self.com1 = torch.zeros((pool.n, 3, 64), dtype=torch.float64, device=d)
        self.G = torch.zeros((pool.n, 4, NCELL), dtype=torch.float64, device=d)
        self.gconst = gconst
        self.correct_am_grav = correct_am_grav

    def run(self, gsolve_type=RHO, precision=FP64, stream=None) -> None:
        b = self.batch
        self.ctx.upward(b.dev, self.com1, self.nodes, self.level_start, gsolve_type, stream)
        b.L.zero_()
        b.Lc.zero_()
        b.run(gsolve_type, precision, stream)
        self.ctx.downward(b.dev, self.com1, self.nodes, self.level_start, b.L, b.Lc, self.G, self.gconst,
                          self.correct_am_grav, gsolve_type, stream)

    def results(self):
        """(L, L_c, G) as numpy arrays after checking the device error flag."""
        self.ctx.batch_status()
        return self.batch.L.cpu().numpy(), self.batch.Lc.cpu().numpy(), self.G.cpu().numpy()


def _host_ptr(a):
    """Pointer of a host buffer (numpy array or CPU torch tensor)."""
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        if a.is_cuda:
            raise ValueError("host buffers expected")
        return ctypes.c_void_p(a.data_ptr())
    if not a.flags.c_contiguous:
        raise ValueError("host buffers must be C-contiguous")
    return ctypes.c_void_p(a.ctypes.data)


class Plan:
    """A batched solve captured into a CUDA graph; launch() replays it."""

    @classmethod
    def from_host(cls, ctx: Context, M, com, mon, is_leaf, n_subgrids: int, items, n_items: int, L, Lc,
                  gsolve_type=RHO, precision=FP64) -> "Plan":
        self = cls.__new__(cls)
        self.ctx = ctx
        self._keep = (M, com, mon, is_leaf, items, L, Lc)   # the graph binds these host pointers
        hp = _host_ptr
        h = ctypes.c_void_p()
        _check(load_library().otfmm_plan_create_host(ctx.handle, hp(M), hp(com), hp(mon), hp(is_leaf),
                                                     ctypes.c_int32(n_subgrids), hp(items), ctypes.c_int32(n_items),
                                                     hp(L), hp(Lc), int(gsolve_type), precision_code(precision),
                                                     ctypes.byref(h)))
        self.handle = h
        return self

    def __init__(self, ctx: Context, dev: DevicePool, items_dev, n_items: int, L, Lc, gsolve_type=RHO,
                 precision=FP64):
        self.ctx = ctx
        self._keep = (dev, items_dev, L, Lc)   # the graph binds these device pointers
        h = ctypes.c_void_p()
        _check(load_library().otfmm_plan_create(ctx.handle, _ptr(dev.M), _ptr(dev.com), _ptr(dev.mon),
                                                _ptr(dev.is_leaf), ctypes.c_int32(dev.n), _ptr(items_dev),
                                                ctypes.c_int32(n_items), _ptr(L), _ptr(Lc), int(gsolve_type),
                                                precision_code(precision), ctypes.byref(h)))
        self.handle = h

    def launch(self, stream=None) -> None:
        _check(load_library().otfmm_plan_launch(self.handle, _stream(stream)))

    def status(self, stream=None) -> None:
        _check(load_library().otfmm_plan_status(self.handle, _stream(stream)))

    def close(self) -> None:
        if getattr(self, "handle", None):
            load_library().otfmm_plan_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


P2M_SLAB_STRIDE_MAX = 8 * 8 * 5 + 19


class PerSubgridSolver:
    """The reference's call pattern on the GPU: one call of the per-subgrid
    entry points per node (multipole_kernel_interface -> otfmm_m2l_soa for
    refined nodes; monopole_kernel_interface -> otfmm_p2p_soa, then
    otfmm_p2m_soa per refined neighbour, for leaves), launched round-robin
    over a pool of streams like the reference's stream pool. The halo buffers
    are staged on the device once at construction (otfmm_stage_soa), so run()
    times the kernels and their launches only."""

    def __init__(self, ctx: Context, pool: SubgridPool, items: np.ndarray, n_streams: int = 32):
        torch = _require_cuda()
        self.ctx = ctx
        self.dev = DevicePool.upload(pool, ctx.device)
        d = torch.device("cuda", ctx.device)
        items = np.ascontiguousarray(items)
        validate_work_list(items, pool.n)
        self.items = items
        kinds = items["kind"]
        self.mpole = np.nonzero(kinds != 2)[0]
        self.leaves = np.nonzero(kinds == 2)[0]
        nm, nl = len(self.mpole), len(self.leaves)
        f64 = dict(dtype=torch.float64, device=d)
        self.m_mon = torch.zeros((nm, ENTRIES), **f64)
        self.m_M = torch.zeros((nm, 20 * COMPONENT_LENGTH), **f64)
        self.m_com = torch.zeros((nm, 3 * COMPONENT_LENGTH), **f64)
        self.m_L = torch.zeros((nm, 20 * COMPONENT_LENGTH_UNPADDED), **f64)
        self.m_Lc = torch.zeros((nm, 3 * COMPONENT_LENGTH_UNPADDED), **f64)
        self.l_mon = torch.zeros((nl, ENTRIES), **f64)
        self.l_icom = torch.zeros((nl, 3, COMPONENT_LENGTH_UNPADDED), **f64)
        self.l_L4 = torch.zeros((nl, 4 * COMPONENT_LENGTH_UNPADDED), **f64)
        self.l_Lc = torch.zeros((nl, 3 * COMPONENT_LENGTH_UNPADDED), **f64)
        self.p2m = []   # (leaf slot, direction, slab index)
        for k, i in enumerate(self.leaves):
            nbs = items[i]["neighbors"]
            for dd in range(26):
                nb = int(nbs[dd])
                if nb >= 0 and not pool.is_leaf[nb]:
                    self.p2m.append((k, dd, nb))
        ns = max(1, len(self.p2m))
        self.s_M = torch.zeros((ns, 20 * P2M_SLAB_STRIDE_MAX), **f64)
        self.s_com = torch.zeros((ns, 3 * P2M_SLAB_STRIDE_MAX), **f64)
        for k, i in enumerate(self.mpole):
            ctx.stage_soa(self.dev, items[i], self.m_mon[k], self.m_M[k], self.m_com[k])
        for k, i in enumerate(self.leaves):
            ctx.stage_soa(self.dev, items[i], self.l_mon[k])
            self.l_icom[k, :, :NCELL] = self.dev.com[int(items[i]["subgrid"])]
        self.p2m_by_leaf = [[] for _ in range(nl)]
        for j, (k, dd, nb) in enumerate(self.p2m):
            ctx.stage_p2m_soa(self.dev, nb, dd, self.s_M[j], self.s_com[j])
            self.p2m_by_leaf[k].append((j, dd))
        self.streams = [torch.cuda.Stream(device=d) for _ in range(n_streams)]
        torch.cuda.synchronize(d)

    def run(self, gsolve_type=RHO, precision=FP64) -> None:
        """Every node's calls, round-robin over the stream pool; the calling
        stream waits for all of them."""
        torch = _require_cuda()
        main = torch.cuda.current_stream()
        start = torch.cuda.Event()
        start.record(main)
        for st in self.streams:
            st.wait_event(start)
        ns = len(self.streams)
        for k, i in enumerate(self.mpole):
            root = int(self.items[i]["kind"]) == 1
            self.ctx.m2l_soa(None if root else self.m_mon[k], self.m_M[k], self.m_com[k], self.m_L[k], self.m_Lc[k],
                             gsolve_type, root, precision, self.streams[k % ns])
        off = len(self.mpole)
        for k, i in enumerate(self.leaves):
            st = self.streams[(off + k) % ns]
            self.ctx.p2p_soa(self.l_mon[k], float(self.items[i]["dx"]), self.l_L4[k], precision, st)
            first = True
            for j, dd in self.p2m_by_leaf[k]:
                self.ctx.p2m_soa(dd, self.s_M[j], self.s_com[j], self.l_icom[k], self.l_L4[k], self.l_Lc[k],
                                 gsolve_type, first, precision, st)
                first = False
        for st in self.streams:
            ev = torch.cuda.Event()
            ev.record(st)
            main.wait_event(ev)

    @property
    def n_launches(self) -> int:
        return len(self.mpole) + len(self.leaves) + len(self.p2m)

    def results(self):
        """L [n, 20, 512] and L_c [n, 3, 512] per subgrid, as the batched path writes them."""
        n = self.dev.n
        L = np.zeros((n, 20, NCELL))
        Lc = np.zeros((n, 3, NCELL))
        mL = self.m_L.cpu().numpy().reshape(-1, 20, COMPONENT_LENGTH_UNPADDED)[:, :, :NCELL]
        mLc = self.m_Lc.cpu().numpy().reshape(-1, 3, COMPONENT_LENGTH_UNPADDED)[:, :, :NCELL]
        sub = self.items["subgrid"]
        L[sub[self.mpole]] = mL
        Lc[sub[self.mpole]] = mLc
        l4 = self.l_L4.cpu().numpy().reshape(-1, 4, COMPONENT_LENGTH_UNPADDED)[:, :, :NCELL]
        lc = self.l_Lc.cpu().numpy().reshape(-1, 3, COMPONENT_LENGTH_UNPADDED)[:, :, :NCELL]
        L[sub[self.leaves], :4] = l4
        has_p2m = np.array([len(x) > 0 for x in self.p2m_by_leaf], dtype=bool)
        Lc[sub[self.leaves][has_p2m]] = lc[has_p2m]
        return L, Lc


PASS_LIB_PATH = Path(__file__).resolve().parent / "libotfmm_adapter_pass.so"


def adapter_pass(ctx: Context, pool: SubgridPool, items: np.ndarray, gsolve_type=RHO, precision=FP64,
                 aggregate: bool = True, threads: int = 8, max_subgrids: int = 2048, max_items: int = 1024,
                 idle_us: int = 200, passes: int = 1, in_place: bool = True, calls_in_flight: int = 64,
                 poll: bool = False):
    """One or more passes over a work list through the C++ drop-in adapter,
    driven like node_server::compute_fmm (one call per node from `threads`
    host threads, AoS inputs; libotfmm_adapter_pass.so). aggregate: the
    aggregated interfaces (otfmm_aggregator) instead of one host-buffer call
    per node. in_place: the batch adds the results into the grids' cells
    itself (otfmm_aggregator_submit_aos), else finish() applies SoA results.
    calls_in_flight: aggregated calls a thread submits before it finishes
    them (HPX suspends a task that waits on its future and runs other nodes'
    tasks, so a solve's calls can all be in flight at once). poll: threads
    poll their calls (otfmm_octotiger::ready) and yield in between instead of
    blocking in finish() (results in place). Returns (L [n,20,512], L_c [n,3,512], seconds per pass)."""
    load_library()
    if not PASS_LIB_PATH.exists():
        raise FileNotFoundError(f"{PASS_LIB_PATH} not built: run `python -m octotiger_b200.build`")
    lib = ctypes.CDLL(str(PASS_LIB_PATH))
    i32, vp = ctypes.c_int32, ctypes.c_void_p
    lib.otfmm_adapter_pass.argtypes = [vp, i32, vp, vp, vp, vp, vp, i32, ctypes.c_int, ctypes.c_int, i32, i32, i32,
                                       i32, i32, i32, i32, vp, vp, vp]
    pool.validate()
    validate_work_list(items, pool.n)
    items = np.ascontiguousarray(items)
    M, com, mon, leaf = (np.ascontiguousarray(getattr(pool, k)) for k in ("M", "com", "mon", "is_leaf"))
    L = np.zeros((pool.n, 20, NCELL))
    Lc = np.zeros((pool.n, 3, NCELL))
    sec = np.zeros(passes)
    _check(lib.otfmm_adapter_pass(ctx.handle, pool.n, M.ctypes.data, com.ctypes.data, mon.ctypes.data,
                                  leaf.ctypes.data, items.ctypes.data, len(items), int(gsolve_type),
                                  precision_code(precision), (3 if poll else 1 if in_place else 2) if aggregate else 0, threads, max_subgrids, max_items,
                                  idle_us, passes, calls_in_flight, L.ctypes.data, Lc.ctypes.data, sec.ctypes.data))
    return L, Lc, sec


def build_info() -> str:
    return load_library().otfmm_build_info().decode()


def measure_fma_peaks(device: int = 0) -> tuple[float, float]:
    _require_cuda()
    a, b = ctypes.c_double(), ctypes.c_double()
    _check(load_library().otfmm_measure_fma_peaks(int(device), ctypes.byref(a), ctypes.byref(b)))
    return a.value, b.value
