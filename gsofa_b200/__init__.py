"""gsofa_b200 -- B200-native symbolic LU factorization (gSoFa's fill traversal).

Python face of ``libgsofa.so`` (C ABI in ``include/gsofa.h``).  It mirrors the
reference's interface for this path:

* :func:`symbfact_min_id` -- the reference's host entry
  ``symbfact_min_id(args, argv, myrank, fill_count, time)``
  (without_space_optimization/symbfact.cuh:991) with the same argv contract;
  it returns ``(fill_count, time_ms)`` and raises :class:`GsofaError` where the
  reference would call ``exit()``.
* :class:`Context` -- device context with device-resident matrices,
  :meth:`Context.symbfact` for one matrix and :meth:`Context.symbfact_batch`
  for many matrices in one persistent launch.

All computation runs in the CUDA library; there is no CPU fallback.  Loading
fails loudly when ``libgsofa.so`` has not been built.
"""
from __future__ import annotations

import ctypes
import dataclasses
import os
from typing import List, Optional, Sequence

import numpy as np

from .matgen import Graph

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libgsofa.so")

OK = 0
STATUS_NAMES = {
    0: "ok", 1: "invalid input", 2: "out of memory", 3: "queue or pattern pool overflow",
    4: "device wait timed out", 5: "CUDA error", 6: "input file error",
    7: "unsupported device or size", 8: "no room for the request now",
}
BUSY = 8

FLAG_NO_DOWNLOAD = 0x1
FLAG_DEVICE_TIMING = 0x2
FLAG_GRAPH = 0x4
FLAG_GLOBAL_STATE = 0x8    # visited bitmaps in global memory (many traversals per SM, any n)
FLAG_SHARED_STATE = 0x10   # visited bitmaps in shared memory (at most two per SM)
FLAG_DIRECT_HOST = 0x20    # symbfact_ranges into host memory: the kernel writes it directly
FLAG_WIDE_REGS = 0x40      # paired passes in 512-thread CTAs with up to 128 registers a thread


class GsofaError(RuntimeError):
    def __init__(self, status: int, what: str = ""):
        self.status = int(status)
        msg = STATUS_NAMES.get(self.status, f"status {status}")
        super().__init__(f"{what}: {msg}" if what else msg)


class Params(ctypes.Structure):
    """gsofa_params; zero fields mean 'choose automatically'."""

    _fields_ = [
        ("src_chunk", ctypes.c_int32),
        ("block_size", ctypes.c_int32),
        ("threads_per_source", ctypes.c_int32),
        ("ctas_per_sm", ctypes.c_int32),
        ("queue_capacity", ctypes.c_int64),
        ("pool_capacity", ctypes.c_int64),
        ("max_supernode_size", ctypes.c_int32),
        ("want_pattern", ctypes.c_int32),
        ("reuse", ctypes.c_int32),
        ("flags", ctypes.c_int32),
        ("part_count", ctypes.c_int32),
        ("part_index", ctypes.c_int32),
        ("line_lo", ctypes.c_int32),
        ("line_hi", ctypes.c_int32),
    ]

    @classmethod
    def default(cls, **kw) -> "Params":
        p = cls()
        lib().gsofa_default_params(ctypes.byref(p))
        for k, v in kw.items():
            if not hasattr(p, k):
                raise TypeError(f"unknown parameter {k!r}")
            setattr(p, k, int(v))
        return p


_i32p = ctypes.POINTER(ctypes.c_int32)
_i64p = ctypes.POINTER(ctypes.c_int64)


class ServerConfig(ctypes.Structure):
    """gsofa_server_config; zero fields mean 'choose automatically'."""

    _fields_ = [
        ("device", ctypes.c_int32),
        ("max_n", ctypes.c_int32),
        ("mem_budget_bytes", ctypes.c_int64),
        ("max_supernode_size", ctypes.c_int32),
        ("src_chunk", ctypes.c_int32),
        ("max_requests", ctypes.c_int32),
        ("idle_exit_us", ctypes.c_int32),
        ("max_n_out", ctypes.c_int32),
        ("flags", ctypes.c_int32),
    ]


class _CResult(ctypes.Structure):
    _fields_ = [
        ("n", ctypes.c_int32),
        ("n_supernodes", ctypes.c_int32),
        ("fill_count", ctypes.c_uint64),
        ("nnz_lu", ctypes.c_uint64),
        ("nnz_u", ctypes.c_uint64),
        ("nnz_l", ctypes.c_uint64),
        ("edges_inspected", ctypes.c_uint64),
        ("sources", ctypes.c_uint64),
        ("x_total", ctypes.c_uint64),
        ("e_insp", ctypes.c_uint64),
        ("levels", ctypes.c_uint64),
        ("reused_sources", ctypes.c_uint64),
        ("cycles", ctypes.c_uint64 * 7),
        ("ctas", ctypes.c_uint64),
        ("kernel_ms", ctypes.c_double),
        ("u_row_count", _i32p),
        ("l_col_count", _i32p),
        ("l_row_count", _i32p),
        ("sn_start", _i32p),
        ("line_flags", ctypes.POINTER(ctypes.c_uint8)),
        ("u_ptr", _i64p),
        ("u_idx", _i32p),
        ("l_ptr", _i64p),
        ("l_idx", _i32p),
        ("internal", ctypes.c_void_p),
        ("u_beg", _i64p),
        ("l_beg", _i64p),
        ("pool_used", ctypes.c_int64),
    ]


@dataclasses.dataclass
class Result:
    """One factorization: counts, supernodes and (optionally) the pattern.

    ``u_ptr/u_idx``: U by rows (sorted columns > s of row s).
    ``l_ptr/l_idx``: L by columns (sorted rows > j of column j).
    """

    n: int
    fill_count: int
    nnz_lu: int
    nnz_u: int
    nnz_l: int
    n_supernodes: int
    edges_inspected: int
    sources: int
    x_total: int
    e_insp: int
    kernel_ms: float
    levels: int = 0
    reused_sources: int = 0
    cycles: tuple = (0, 0, 0, 0, 0, 0, 0)
    ctas: int = 0
    u_row_count: Optional[np.ndarray] = None
    l_col_count: Optional[np.ndarray] = None
    l_row_count: Optional[np.ndarray] = None
    sn_start: Optional[np.ndarray] = None
    line_flags: Optional[np.ndarray] = None
    u_ptr: Optional[np.ndarray] = None
    u_idx: Optional[np.ndarray] = None
    l_ptr: Optional[np.ndarray] = None
    l_idx: Optional[np.ndarray] = None
    # ranges form (Context.symbfact_ranges): U row s = pool[u_beg[s] :
    # u_beg[s] + u_row_count[s]], L column j = pool[l_beg[j] : ...]
    u_beg: Optional[np.ndarray] = None
    l_beg: Optional[np.ndarray] = None
    pool_used: int = 0
    pool: Optional[np.ndarray] = None

    def u_row(self, s: int) -> np.ndarray:
        """Sorted columns > s of U row s (either pattern form)."""
        if self.u_ptr is not None:
            return self.u_idx[self.u_ptr[s]:self.u_ptr[s + 1]]
        b = int(self.u_beg[s])
        return self.pool[b:b + int(self.u_row_count[s])]

    def l_col(self, j: int) -> np.ndarray:
        """Sorted rows > j of L column j (either pattern form)."""
        if self.l_ptr is not None:
            return self.l_idx[self.l_ptr[j]:self.l_ptr[j + 1]]
        b = int(self.l_beg[j])
        return self.pool[b:b + int(self.l_col_count[j])]


_lib = None


def lib():
    """Loads libgsofa.so; raises when it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing; build it with `python -m gsofa_b200.build`")
    L = ctypes.CDLL(LIB_PATH)
    vp = ctypes.c_void_p
    L.gsofa_status_str.argtypes = [ctypes.c_int]
    L.gsofa_status_str.restype = ctypes.c_char_p
    L.gsofa_abi_version.restype = ctypes.c_int
    L.gsofa_default_params.argtypes = [ctypes.POINTER(Params)]
    L.gsofa_default_params.restype = None
    L.gsofa_create.argtypes = [ctypes.POINTER(vp), ctypes.c_int, ctypes.c_size_t]
    L.gsofa_create.restype = ctypes.c_int
    L.gsofa_destroy.argtypes = [vp]
    L.gsofa_destroy.restype = None
    L.gsofa_set_stream.argtypes = [vp, vp]
    L.gsofa_set_stream.restype = ctypes.c_int
    L.gsofa_read_text.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p,
                                  _i32p, _i64p, ctypes.POINTER(_i32p), ctypes.POINTER(_i32p),
                                  ctypes.POINTER(_i32p)]
    L.gsofa_read_text.restype = ctypes.c_int
    L.gsofa_result_supernodal.argtypes = [vp, ctypes.POINTER(_CResult), ctypes.POINTER(_CSupernodal)]
    L.gsofa_result_supernodal.restype = ctypes.c_int
    L.gsofa_supernodal_free.argtypes = [ctypes.POINTER(_CSupernodal)]
    L.gsofa_supernodal_free.restype = None
    L.gsofa_result_supernodal_sizes.argtypes = [vp, ctypes.POINTER(_CResult), ctypes.POINTER(ctypes.c_int32),
                                                _i64p, _i64p]
    L.gsofa_result_supernodal_sizes.restype = ctypes.c_int
    L.gsofa_result_supernodal_fetch.argtypes = [vp, ctypes.POINTER(_CResult), _i32p, _i32p, _i64p, _i32p,
                                                _i64p, _i32p]
    L.gsofa_result_supernodal_fetch.restype = ctypes.c_int
    L.gsofa_write_binary.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int32,
                                     ctypes.c_int64, _i32p, _i32p, _i32p]
    L.gsofa_write_binary.restype = ctypes.c_int
    L.gsofa_free.argtypes = [vp]
    L.gsofa_free.restype = None
    L.gsofa_upload.argtypes = [vp, ctypes.c_int32, ctypes.c_int64, _i32p, _i32p, _i32p,
                               ctypes.POINTER(vp)]
    L.gsofa_upload.restype = ctypes.c_int
    L.gsofa_matrix_free.argtypes = [vp]
    L.gsofa_matrix_free.restype = None
    L.gsofa_matrix_n.argtypes = [vp]
    L.gsofa_matrix_n.restype = ctypes.c_int32
    L.gsofa_symbfact.argtypes = [vp, vp, ctypes.POINTER(Params), ctypes.POINTER(_CResult)]
    L.gsofa_symbfact.restype = ctypes.c_int
    L.gsofa_symbfact_batch.argtypes = [vp, ctypes.c_int, ctypes.POINTER(vp), ctypes.POINTER(Params),
                                       ctypes.POINTER(_CResult)]
    L.gsofa_symbfact_batch.restype = ctypes.c_int
    L.gsofa_result_free.argtypes = [ctypes.POINTER(_CResult)]
    L.gsofa_result_free.restype = None
    L.gsofa_result_fetch.argtypes = [vp, ctypes.POINTER(_CResult), _i32p, _i32p, _i32p, _i32p,
                                     _i64p, _i32p, _i64p, _i32p]
    L.gsofa_result_fetch.restype = ctypes.c_int
    L.gsofa_symbfact_ranges.argtypes = [vp, ctypes.c_int, ctypes.POINTER(vp), ctypes.POINTER(Params),
                                        vp, ctypes.c_int64, ctypes.POINTER(_CResult)]
    L.gsofa_symbfact_ranges.restype = ctypes.c_int
    L.gsofa_result_fetch_ranges.argtypes = [vp, ctypes.POINTER(_CResult), _i64p, _i64p]
    L.gsofa_result_fetch_ranges.restype = ctypes.c_int
    L.gsofa_symbfact_counts_noalloc.argtypes = [ctypes.c_int, vp, ctypes.c_int32, ctypes.c_int64,
                                                vp, vp, vp, ctypes.c_int32, vp, vp, vp,
                                                ctypes.POINTER(ctypes.c_uint64)]
    L.gsofa_symbfact_counts_noalloc.restype = ctypes.c_int
    L.gsofa_predict_line_counts.argtypes = [ctypes.c_int32, ctypes.c_int64, _i32p, _i32p, _i32p, _i64p]
    L.gsofa_predict_line_counts.restype = ctypes.c_int
    L.gsofa_partition_lines.argtypes = [ctypes.c_int32, ctypes.c_int64, _i32p, _i32p, _i32p, ctypes.c_int32,
                                        _i32p, ctypes.POINTER(ctypes.c_double)]
    L.gsofa_partition_lines.restype = ctypes.c_int
    L.gsofa_order_rcm.argtypes = [vp, ctypes.c_int32, ctypes.c_int64, _i32p, _i32p, _i32p, _i32p]
    L.gsofa_order_rcm.restype = ctypes.c_int
    L.gsofa_permute_lines.argtypes = [ctypes.c_int32, ctypes.c_int64, _i32p, _i32p, _i32p, _i32p, _i32p, _i32p,
                                      _i32p]
    L.gsofa_permute_lines.restype = ctypes.c_int
    L.gsofa_supernodes_from_lines.argtypes = [ctypes.c_int32, _i32p, ctypes.POINTER(ctypes.c_uint8),
                                              ctypes.c_int32, _i32p]
    L.gsofa_supernodes_from_lines.restype = ctypes.c_int32
    L.gsofa_server_create.argtypes = [ctypes.POINTER(vp), ctypes.POINTER(ServerConfig)]
    L.gsofa_server_create.restype = ctypes.c_int
    L.gsofa_server_destroy.argtypes = [vp]
    L.gsofa_server_destroy.restype = None
    L.gsofa_server_drain.argtypes = [vp]
    L.gsofa_server_drain.restype = ctypes.c_int
    L.gsofa_server_request_bytes.argtypes = [vp, ctypes.c_int32, ctypes.c_int64]
    L.gsofa_server_request_bytes.restype = ctypes.c_size_t
    L.gsofa_server_submit.argtypes = [vp, ctypes.c_int32, ctypes.c_int64, _i32p, _i32p, _i32p,
                                      ctypes.POINTER(ctypes.c_int64)]
    L.gsofa_server_submit.restype = ctypes.c_int
    L.gsofa_server_poll.argtypes = [vp, ctypes.POINTER(ctypes.c_int64), ctypes.c_int32,
                                    ctypes.POINTER(ctypes.c_int32)]
    L.gsofa_server_poll.restype = ctypes.c_int
    L.gsofa_server_result.argtypes = [vp, ctypes.c_int64, ctypes.POINTER(_CResult)]
    L.gsofa_server_result.restype = ctypes.c_int
    L.gsofa_predict_scratch_bytes.argtypes = [vp, ctypes.c_int32, ctypes.c_int64, ctypes.POINTER(Params)]
    L.gsofa_predict_scratch_bytes.restype = ctypes.c_size_t
    L.gsofa_symbfact_min_id.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_char_p), ctypes.c_int,
                                        ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_double)]
    L.gsofa_symbfact_min_id.restype = ctypes.c_int
    _lib = L
    return L


def _check(status: int, what: str = "") -> None:
    if status != OK:
        raise GsofaError(status, what)


class _CSupernodal(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int32), ("nsuper", ctypes.c_int32), ("nlsub", ctypes.c_int64),
                ("nusub", ctypes.c_int64), ("xsup", _i32p), ("supno", _i32p), ("xlsub", _i64p),
                ("lsub", _i32p), ("xusub", _i64p), ("usub", _i32p)]


@dataclasses.dataclass
class Supernodal:
    """SuperLU-style supernodal structure (gsofa_result_supernodal): supernode
    k holds columns xsup[k] .. xsup[k+1]-1; its rows are lsub[xlsub[k] ..
    xlsub[k+1]) (the diagonal block, then the rows below it of its last
    column), its columns right of the block usub[xusub[k] .. xusub[k+1])."""
    n: int
    nsuper: int
    xsup: np.ndarray
    supno: np.ndarray
    xlsub: np.ndarray
    lsub: np.ndarray
    xusub: np.ndarray
    usub: np.ndarray


def _arr(ptr, count: int, dtype) -> Optional[np.ndarray]:
    if not ptr or count < 0:
        return None
    if count == 0:
        return np.zeros(0, dtype)
    return np.ctypeslib.as_array(ptr, shape=(count,)).astype(dtype, copy=True)


def _convert(r: _CResult) -> Result:
    n = int(r.n)
    out = Result(n=n, fill_count=int(r.fill_count), nnz_lu=int(r.nnz_lu), nnz_u=int(r.nnz_u),
                 nnz_l=int(r.nnz_l), n_supernodes=int(r.n_supernodes),
                 edges_inspected=int(r.edges_inspected), sources=int(r.sources),
                 x_total=int(r.x_total), e_insp=int(r.e_insp), kernel_ms=float(r.kernel_ms),
                 levels=int(r.levels), reused_sources=int(r.reused_sources),
                 cycles=tuple(int(c) for c in r.cycles), ctas=int(r.ctas))
    out.u_row_count = _arr(r.u_row_count, n, np.int32)
    out.l_col_count = _arr(r.l_col_count, n, np.int32)
    out.l_row_count = _arr(r.l_row_count, n, np.int32)
    out.sn_start = _arr(r.sn_start, int(r.n_supernodes), np.int32)
    out.line_flags = _arr(r.line_flags, n, np.uint8)
    out.u_ptr = _arr(r.u_ptr, n + 1, np.int64)
    out.l_ptr = _arr(r.l_ptr, n + 1, np.int64)
    out.u_idx = _arr(r.u_idx, int(r.nnz_u), np.int32)
    out.l_idx = _arr(r.l_idx, int(r.nnz_l), np.int32)
    out.u_beg = _arr(r.u_beg, n, np.int64)
    out.l_beg = _arr(r.l_beg, n, np.int64)
    out.pool_used = int(r.pool_used)
    return out


class Matrix:
    """A device-resident matrix (G and its transpose) owned by a Context."""

    def __init__(self, ctx: "Context", handle: ctypes.c_void_p, n: int, nnz: int):
        self._ctx = ctx
        self._h = handle
        self.n = n
        self.nnz = nnz

    def free(self) -> None:
        if self._h:
            lib().gsofa_matrix_free(self._h)
            self._h = None
            mats = self._ctx._mats
            if mats and mats[-1] is self:
                mats.pop()
            elif self in mats:
                mats.remove(self)

    def __enter__(self) -> "Matrix":
        return self

    def __exit__(self, *exc) -> None:
        self.free()

    @property
    def handle(self):
        if not self._h:
            raise GsofaError(1, "matrix already freed")
        return self._h


class Context:
    """A device context: stream, scratch pools and uploaded matrices."""

    def __init__(self, device: int = 0, mem_budget_bytes: int = 0):
        h = ctypes.c_void_p()
        _check(lib().gsofa_create(ctypes.byref(h), int(device), int(mem_budget_bytes)), "gsofa_create")
        self._h = h
        self._mats: List[Matrix] = []

    def set_stream(self, cuda_stream: int) -> None:
        """Issue work on this cudaStream_t handle (0: the context's own)."""
        _check(lib().gsofa_set_stream(self._h, ctypes.c_void_p(int(cuda_stream) or None)), "gsofa_set_stream")

    def close(self) -> None:
        if self._h:
            for m in self._mats:
                m._h = None
            lib().gsofa_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def upload(self, beg, end=None, adj=None) -> Matrix:
        """Uploads a matrix given as a Graph or as (beg, end, adj) int32 arrays."""
        if isinstance(beg, Graph):
            g = beg
            beg, end, adj = g.beg, g.end, g.adj
        beg = np.ascontiguousarray(beg, dtype=np.int32)
        end = np.ascontiguousarray(end, dtype=np.int32)
        adj = np.ascontiguousarray(adj, dtype=np.int32)
        if beg.shape != end.shape:
            raise GsofaError(1, "beg and end differ in length")
        h = ctypes.c_void_p()
        _check(lib().gsofa_upload(self._h, beg.shape[0], adj.shape[0], beg.ctypes.data_as(_i32p),
                                  end.ctypes.data_as(_i32p), adj.ctypes.data_as(_i32p),
                                  ctypes.byref(h)), "gsofa_upload")
        m = Matrix(self, h, int(beg.shape[0]), int(adj.shape[0]))
        self._mats.append(m)
        return m

    def order_rcm(self, g: Graph) -> np.ndarray:
        """Reverse Cuthill-McKee order of A + A^T computed on the GPU
        (gsofa_order_rcm): perm[new] = old, int32[n]."""
        beg = np.ascontiguousarray(g.beg, dtype=np.int32)
        end = np.ascontiguousarray(g.end, dtype=np.int32)
        adj = np.ascontiguousarray(g.adj if g.nnz else np.zeros(1, np.int32), dtype=np.int32)
        perm = np.zeros(max(g.n, 1), np.int32)
        _check(lib().gsofa_order_rcm(self._h, int(g.n), int(g.nnz), beg.ctypes.data_as(_i32p),
                                     end.ctypes.data_as(_i32p), adj.ctypes.data_as(_i32p),
                                     perm.ctypes.data_as(_i32p)), "gsofa_order_rcm")
        return perm[:g.n]

    def symbfact(self, m: Matrix, params: Optional[Params] = None, **kw) -> Result:
        p = params if params is not None else Params.default(**kw)
        r = _CResult()
        _check(lib().gsofa_symbfact(self._h, m.handle, ctypes.byref(p), ctypes.byref(r)), "gsofa_symbfact")
        try:
            return _convert(r)
        finally:
            lib().gsofa_result_free(ctypes.byref(r))

    def symbfact_supernodal(self, m: Matrix, params: Optional[Params] = None, out: Optional[dict] = None,
                            **kw):
        """Factorizes with the pattern kept on the device and returns
        (Result without per-line arrays, Supernodal): only the compact
        supernodal structure crosses PCIe, not the pattern.  `out` may hold
        caller-owned buffers (e.g. views of page-locked memory) named like the
        Supernodal fields; the returned arrays are then views of them."""
        p = Params()
        ctypes.pointer(p)[0] = params if params is not None else Params.default(**kw)
        p.want_pattern = 1
        p.flags |= FLAG_NO_DOWNLOAD
        r = _CResult()
        _check(lib().gsofa_symbfact(self._h, m.handle, ctypes.byref(p), ctypes.byref(r)), "gsofa_symbfact")
        try:
            res = _convert(r)
            return res, self._supernodal_of(r, res.n, out)
        finally:
            lib().gsofa_result_free(ctypes.byref(r))

    def _supernodal_of(self, r: "_CResult", n: int, out: Optional[dict]) -> "Supernodal":
        """The supernodal structure of the C result r (last job on this
        context, made with the pattern) into new or caller buffers."""
        ns, nl, nu = ctypes.c_int32(), ctypes.c_int64(), ctypes.c_int64()
        _check(lib().gsofa_result_supernodal_sizes(self._h, ctypes.byref(r), ctypes.byref(ns),
                                                   ctypes.byref(nl), ctypes.byref(nu)),
               "gsofa_result_supernodal_sizes")
        k = ns.value
        need = {"xsup": (k + 1, np.int32), "supno": (n, np.int32), "xlsub": (k + 1, np.int64),
                "lsub": (nl.value, np.int32), "xusub": (k + 1, np.int64), "usub": (nu.value, np.int32)}
        bufs = {}
        for key, (cnt, dt) in need.items():
            b = None if out is None else out.get(key)
            if b is None:
                b = np.empty(max(cnt, 1), dt)
            elif b.shape[0] < cnt or b.dtype != dt:
                raise GsofaError(1, f"buffer {key} holds {b.shape[0]} {b.dtype} < {cnt} {np.dtype(dt)}")
            bufs[key] = b
        ptr = lambda key: bufs[key].ctypes.data_as(_i64p if key.startswith("x") and key != "xsup"  # noqa: E731
                                                    else _i32p)
        _check(lib().gsofa_result_supernodal_fetch(self._h, ctypes.byref(r), ptr("xsup"), ptr("supno"),
                                                   ptr("xlsub"), ptr("lsub"), ptr("xusub"), ptr("usub")),
               "gsofa_result_supernodal_fetch")
        return Supernodal(n, k, *(bufs[key][:cnt] for key, (cnt, _) in need.items()))

    def symbfact_into(self, m: Matrix, params: Params, out: dict) -> Result:
        """Factorizes and copies every result array into caller-owned host
        buffers (numpy arrays, e.g. views of page-locked memory) named like
        the Result fields; returns the Result with those arrays (trimmed)."""
        p = Params()
        ctypes.pointer(p)[0] = params
        p.flags |= FLAG_NO_DOWNLOAD
        r = _CResult()
        _check(lib().gsofa_symbfact(self._h, m.handle, ctypes.byref(p), ctypes.byref(r)), "gsofa_symbfact")
        try:
            res = _convert(r)
            need = {"u_row_count": r.n, "l_col_count": r.n, "l_row_count": r.n if p.want_pattern else 0,
                    "sn_start": r.n_supernodes, "u_ptr": r.n + 1, "l_ptr": r.n + 1,
                    "u_idx": r.nnz_u if p.want_pattern else 0, "l_idx": r.nnz_l if p.want_pattern else 0}
            ptrs = {}
            for k, cnt in need.items():
                buf = out.get(k)
                if buf is None or cnt == 0 or (k in ("u_ptr", "l_ptr", "u_idx", "l_idx") and not p.want_pattern):
                    ptrs[k] = None
                    continue
                if buf.shape[0] < cnt:
                    raise GsofaError(1, f"buffer {k} holds {buf.shape[0]} < {cnt}")
                ptrs[k] = buf.ctypes.data_as(_i64p if k.endswith("ptr") else _i32p)
                setattr(res, k, buf[:cnt])
            _check(lib().gsofa_result_fetch(self._h, ctypes.byref(r), ptrs["u_row_count"], ptrs["l_col_count"],
                                            ptrs["l_row_count"], ptrs["sn_start"], ptrs["u_ptr"], ptrs["u_idx"],
                                            ptrs["l_ptr"], ptrs["l_idx"]), "gsofa_result_fetch")
            return res
        finally:
            lib().gsofa_result_free(ctypes.byref(r))

    def symbfact_ranges(self, mats, pool, params: Optional[Params] = None, out: Optional[dict] = None,
                        supernodal: bool = False, **kw):
        """The pattern in the reference's begin/end layout, written straight
        into `pool`: a numpy int32 array in page-locked host memory (e.g. a
        view of a pinned torch tensor; the lists then travel to the host
        while the traversals run) or a CUDA int32 torch tensor on this
        context's device.  `mats` is one Matrix or a sequence (one launch).

        Returns a Result (or a list of them) whose u_beg / l_beg index into
        the pool (Result.u_row / l_col read lists back from a host pool).
        Raises GsofaError(3) when the pool is too small; its `needed`
        attribute then holds the entries the job needs.  `out` may hold
        caller buffers for the per-line arrays (u_row_count, l_col_count,
        l_row_count, sn_start, u_beg, l_beg), filled without allocation.
        supernodal=True (one matrix) returns (Result, Supernodal), the
        structure built on the device from the pool."""
        single = isinstance(mats, Matrix)
        ms = [mats] if single else list(mats)
        p = Params()
        ctypes.pointer(p)[0] = params if params is not None else Params.default(**kw)
        p.want_pattern = 2
        if out is not None:
            p.flags |= FLAG_NO_DOWNLOAD
        host = isinstance(pool, np.ndarray)
        if host:
            if pool.dtype != np.int32 or not pool.flags["C_CONTIGUOUS"]:
                raise GsofaError(1, "pool must be a contiguous int32 array")
            addr, cap = pool.ctypes.data, pool.shape[0]
        else:
            if str(getattr(pool, "dtype", "")) != "torch.int32" or not pool.is_contiguous():
                raise GsofaError(1, "pool must be a contiguous int32 tensor")
            addr, cap = pool.data_ptr(), pool.numel()
        k = len(ms)
        hs = (ctypes.c_void_p * k)(*[m.handle for m in ms])
        rs = (_CResult * k)()
        st = lib().gsofa_symbfact_ranges(self._h, k, hs, ctypes.byref(p), ctypes.c_void_p(addr), int(cap), rs)
        if st != OK:
            err = GsofaError(st, "gsofa_symbfact_ranges")
            err.needed = int(rs[0].pool_used)
            raise err
        try:
            res = [_convert(rs[i]) for i in range(k)]
            if out is not None:
                if k != 1:
                    raise GsofaError(1, "caller buffers take one matrix")
                r0 = res[0]
                n = r0.n
                for key, dt in (("u_row_count", np.int32), ("l_col_count", np.int32), ("l_row_count", np.int32),
                                ("sn_start", np.int32), ("u_beg", np.int64), ("l_beg", np.int64)):
                    cnt = r0.n_supernodes if key == "sn_start" else n
                    b = out.get(key)
                    if b is None or b.shape[0] < cnt or b.dtype != dt:
                        raise GsofaError(1, f"buffer {key} missing or smaller than {cnt} {np.dtype(dt)}")
                    setattr(r0, key, b[:cnt])
                _check(lib().gsofa_result_fetch(self._h, ctypes.byref(rs[0]),
                                                out["u_row_count"].ctypes.data_as(_i32p),
                                                out["l_col_count"].ctypes.data_as(_i32p),
                                                out["l_row_count"].ctypes.data_as(_i32p),
                                                out["sn_start"].ctypes.data_as(_i32p), None, None, None, None),
                       "gsofa_result_fetch")
                _check(lib().gsofa_result_fetch_ranges(self._h, ctypes.byref(rs[0]),
                                                       out["u_beg"].ctypes.data_as(_i64p),
                                                       out["l_beg"].ctypes.data_as(_i64p)),
                       "gsofa_result_fetch_ranges")
            for r in res:
                r.pool = pool if host else None
            if supernodal:
                if k != 1:
                    raise GsofaError(1, "the supernodal structure takes one matrix")
                return res[0], self._supernodal_of(rs[0], res[0].n, None)
            return res[0] if single else res
        finally:
            for i in range(k):
                lib().gsofa_result_free(ctypes.byref(rs[i]))

    def symbfact_batch(self, mats: Sequence[Matrix], params: Optional[Params] = None, **kw) -> List[Result]:
        p = params if params is not None else Params.default(**kw)
        k = len(mats)
        hs = (ctypes.c_void_p * k)(*[m.handle for m in mats])
        rs = (_CResult * k)()
        _check(lib().gsofa_symbfact_batch(self._h, k, hs, ctypes.byref(p), rs), "gsofa_symbfact_batch")
        try:
            return [_convert(rs[i]) for i in range(k)]
        finally:
            for i in range(k):
                lib().gsofa_result_free(ctypes.byref(rs[i]))

    def predict_scratch_bytes(self, n: int, nnz: int, params: Optional[Params] = None) -> int:
        p = params if params is not None else Params.default()
        return int(lib().gsofa_predict_scratch_bytes(self._h, int(n), int(nnz), ctypes.byref(p)))


class StreamServer:
    """A persistent-kernel factorization server (continuous batching).

    submit() uploads a matrix and publishes its work to the running kernel;
    it returns None when the request does not fit right now (poll, fetch
    finished results, try again).  poll() lists finished request ids;
    result() returns one (counts, line flags, supernodes, totals) and frees
    its device memory."""

    def __init__(self, device: int = 0, mem_budget_bytes: int = 0, max_n: int = 0,
                 max_supernode_size: int = 0, src_chunk: int = 0, max_requests: int = 0,
                 idle_exit_us: int = 0, flags: int = 0):
        cfg = ServerConfig(device, max_n, mem_budget_bytes, max_supernode_size, src_chunk,
                           max_requests, idle_exit_us, 0, flags)
        h = ctypes.c_void_p()
        _check(lib().gsofa_server_create(ctypes.byref(h), ctypes.byref(cfg)), "gsofa_server_create")
        self._h = h
        self.max_n = int(cfg.max_n_out)
        self._ids = (ctypes.c_int64 * 4096)()

    def close(self) -> None:
        if self._h:
            lib().gsofa_server_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def drain(self) -> None:
        """Waits until every published request is done and the kernel exited."""
        _check(lib().gsofa_server_drain(self._h), "gsofa_server_drain")

    def request_bytes(self, n: int, nnz: int) -> int:
        return int(lib().gsofa_server_request_bytes(self._h, int(n), int(nnz)))

    def submit(self, g: Graph) -> Optional[int]:
        beg = np.ascontiguousarray(g.beg, dtype=np.int32)
        end = np.ascontiguousarray(g.end, dtype=np.int32)
        adj = np.ascontiguousarray(g.adj if g.nnz else np.zeros(1, np.int32), dtype=np.int32)
        rid = ctypes.c_int64()
        st = lib().gsofa_server_submit(self._h, g.n, g.nnz, beg.ctypes.data_as(_i32p), end.ctypes.data_as(_i32p),
                                       adj.ctypes.data_as(_i32p), ctypes.byref(rid))
        if st == BUSY:
            return None
        _check(st, "gsofa_server_submit")
        return int(rid.value)

    def poll(self) -> List[int]:
        cnt = ctypes.c_int32()
        _check(lib().gsofa_server_poll(self._h, self._ids, len(self._ids), ctypes.byref(cnt)), "gsofa_server_poll")
        return [int(self._ids[i]) for i in range(cnt.value)]

    def result(self, rid: int) -> Result:
        r = _CResult()
        _check(lib().gsofa_server_result(self._h, int(rid), ctypes.byref(r)), "gsofa_server_result")
        try:
            return _convert(r)
        finally:
            lib().gsofa_result_free(ctypes.byref(r))


def read_text(beg_file: str, end_file: str, csr_file: str) -> Graph:
    """Reads the reference's colbeg/colend/csr text files (or their binary
    form, see write_binary) through the library."""
    n = ctypes.c_int32()
    nnz = ctypes.c_int64()
    b, e, a = _i32p(), _i32p(), _i32p()
    _check(lib().gsofa_read_text(beg_file.encode(), end_file.encode(), csr_file.encode(),
                                 ctypes.byref(n), ctypes.byref(nnz), ctypes.byref(b), ctypes.byref(e),
                                 ctypes.byref(a)), "gsofa_read_text")
    try:
        g = Graph(int(n.value), _arr(b, n.value, np.int32), _arr(e, n.value, np.int32),
                  _arr(a, nnz.value, np.int32), os.path.basename(csr_file))
    finally:
        for p in (b, e, a):
            lib().gsofa_free(ctypes.cast(p, ctypes.c_void_p))
    return g


def write_binary(g: Graph, beg_file: str, end_file: str, csr_file: str) -> None:
    """Writes g as the three input files in the library's binary form, which
    read_text (and the argv entry) load without text parsing."""
    b = np.ascontiguousarray(g.beg, dtype=np.int32)
    e = np.ascontiguousarray(g.end, dtype=np.int32)
    a = np.ascontiguousarray(g.adj, dtype=np.int32)
    _check(lib().gsofa_write_binary(beg_file.encode(), end_file.encode(), csr_file.encode(), int(g.n),
                                    int(a.shape[0]), b.ctypes.data_as(_i32p), e.ctypes.data_as(_i32p),
                                    a.ctypes.data_as(_i32p)), "gsofa_write_binary")


def symbfact_min_id(argv: Sequence[str], myrank: int = 0):
    """The reference entry point: returns (fill_count, time_ms) for argv
    ``[prog, colbeg, colend, csr, N_GPU, (mem_GB, (max_supernode_size, GPUs_per_node))]``."""
    enc = [str(a).encode() for a in argv]
    arr = (ctypes.c_char_p * len(enc))(*enc)
    fc = ctypes.c_uint64()
    t = ctypes.c_double()
    _check(lib().gsofa_symbfact_min_id(len(enc), arr, int(myrank), ctypes.byref(fc), ctypes.byref(t)),
           "symbfact_min_id")
    return int(fc.value), float(t.value)


NOALLOC_MAX_N = 16384
NOALLOC_MAX_NNZ = 262144


def symbfact_counts_noalloc(device: int, stream: int, n: int, nnz: int, d_beg: int, d_end: int,
                            d_adj: int, d_u_row_count: int, d_l_col_count: int, d_sn_start: int,
                            max_supernode_size: int = 0):
    """Counts-only factorization that allocates no device memory.

    For callers that cannot call cudaMalloc (code living under a host
    framework's own device allocator or memory budget, or on a path where
    cudaMalloc's implicit synchronisation is not allowed).  All arguments are
    raw device addresses (ints) of buffers the caller owns: the
    colbeg/colend/csr triple and outputs of n int32 each.  Scratch comes from
    a static device array inside the library (n <= NOALLOC_MAX_N,
    nnz <= NOALLOC_MAX_NNZ).  Returns (fill_count, nnz_lu, n_supernodes);
    the first n_supernodes entries of the sn_start buffer are the supernode
    starts.  Calls on one device share the scratch, so issue them one at a
    time."""
    summary = (ctypes.c_uint64 * 3)()
    vp = ctypes.c_void_p
    _check(lib().gsofa_symbfact_counts_noalloc(int(device), vp(int(stream) or None), int(n), int(nnz),
                                               vp(d_beg), vp(d_end), vp(d_adj), int(max_supernode_size),
                                               vp(d_u_row_count), vp(d_l_col_count), vp(d_sn_start),
                                               summary), "gsofa_symbfact_counts_noalloc")
    return int(summary[0]), int(summary[1]), int(summary[2])


def partition_lines(g: Graph, parts: int):
    """Contiguous source-line ranges of equal predicted work (host):
    returns (cuts int32[parts+1], predicted work float64[parts]); part p is
    lines [cuts[p], cuts[p+1])."""
    beg = np.ascontiguousarray(g.beg, dtype=np.int32)
    end = np.ascontiguousarray(g.end, dtype=np.int32)
    adj = np.ascontiguousarray(g.adj if g.nnz else np.zeros(1, np.int32), dtype=np.int32)
    cuts = np.zeros(parts + 1, np.int32)
    work = np.zeros(parts, np.float64)
    _check(lib().gsofa_partition_lines(int(g.n), int(g.nnz), beg.ctypes.data_as(_i32p), end.ctypes.data_as(_i32p),
                                       adj.ctypes.data_as(_i32p), int(parts), cuts.ctypes.data_as(_i32p),
                                       work.ctypes.data_as(ctypes.POINTER(ctypes.c_double))),
           "gsofa_partition_lines")
    return cuts, work


def permute_lines(g: Graph, perm) -> Graph:
    """The symmetric permutation P A P^T (gsofa_permute_lines, host): new
    line k is old line perm[k], ids renamed, lines sorted and packed."""
    beg = np.ascontiguousarray(g.beg, dtype=np.int32)
    end = np.ascontiguousarray(g.end, dtype=np.int32)
    adj = np.ascontiguousarray(g.adj if g.nnz else np.zeros(1, np.int32), dtype=np.int32)
    p = np.ascontiguousarray(perm, dtype=np.int32)
    if p.shape != (g.n,):
        raise GsofaError(1, "perm must have n entries")
    total = int((end.astype(np.int64) - beg).sum()) if g.n else 0
    ob = np.zeros(max(g.n, 1), np.int32)
    oe = np.zeros(max(g.n, 1), np.int32)
    oa = np.zeros(max(total, 1), np.int32)
    _check(lib().gsofa_permute_lines(int(g.n), int(g.nnz), beg.ctypes.data_as(_i32p), end.ctypes.data_as(_i32p),
                                     adj.ctypes.data_as(_i32p), p.ctypes.data_as(_i32p), ob.ctypes.data_as(_i32p),
                                     oe.ctypes.data_as(_i32p), oa.ctypes.data_as(_i32p)), "gsofa_permute_lines")
    name = f"{g.name}_perm" if getattr(g, "name", "") else "permuted"
    return Graph(g.n, ob[:g.n], oe[:g.n], oa[:total], name)


def predict_line_counts(g: Graph) -> np.ndarray:
    """Upper bound on every line's |U row| and |L column| from the symmetric
    structure A + A^T (exact for symmetric patterns); host-only."""
    beg = np.ascontiguousarray(g.beg, dtype=np.int32)
    end = np.ascontiguousarray(g.end, dtype=np.int32)
    adj = np.ascontiguousarray(g.adj if g.nnz else np.zeros(1, np.int32), dtype=np.int32)
    out = np.zeros(max(g.n, 1), np.int64)
    _check(lib().gsofa_predict_line_counts(int(g.n), int(g.nnz), beg.ctypes.data_as(_i32p),
                                           end.ctypes.data_as(_i32p), adj.ctypes.data_as(_i32p),
                                           out.ctypes.data_as(_i64p)), "gsofa_predict_line_counts")
    return out[:g.n]


def supernodes_from_lines(u_row_count, line_flags, max_supernode_size: int = 0) -> np.ndarray:
    """Supernode starts from per-line U row counts and link flags (host)."""
    u = np.ascontiguousarray(u_row_count, dtype=np.int32)
    f = np.ascontiguousarray(line_flags, dtype=np.uint8)
    n = u.shape[0]
    out = np.zeros(max(n, 1), np.int32)
    k = lib().gsofa_supernodes_from_lines(n, u.ctypes.data_as(_i32p),
                                          f.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)),
                                          int(max_supernode_size), out.ctypes.data_as(_i32p))
    if k < 0:
        raise GsofaError(1, "gsofa_supernodes_from_lines")
    return out[:k].copy()


def exported_symbols() -> List[str]:
    """Names of the C ABI entry points declared in include/gsofa.h."""
    return ["gsofa_symbfact_min_id", "gsofa_status_str", "gsofa_abi_version", "gsofa_default_params",
            "gsofa_create", "gsofa_destroy", "gsofa_set_stream", "gsofa_read_text", "gsofa_write_binary",
            "gsofa_free", "gsofa_upload",
            "gsofa_matrix_free", "gsofa_matrix_n", "gsofa_symbfact", "gsofa_symbfact_batch",
            "gsofa_result_free", "gsofa_result_fetch", "gsofa_symbfact_ranges", "gsofa_result_fetch_ranges",
            "gsofa_result_supernodal", "gsofa_supernodal_free",
            "gsofa_result_supernodal_sizes", "gsofa_result_supernodal_fetch",
            "gsofa_predict_scratch_bytes",
            "gsofa_symbfact_counts_noalloc", "gsofa_supernodes_from_lines", "gsofa_partition_lines",
            "gsofa_predict_line_counts", "gsofa_order_rcm", "gsofa_permute_lines",
            "gsofa_server_create",
            "gsofa_server_destroy", "gsofa_server_request_bytes", "gsofa_server_submit",
            "gsofa_server_poll", "gsofa_server_result", "gsofa_server_drain"]
