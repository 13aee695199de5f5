"""The host-side mirror of warren-core's compute interface, over the C ABI.

Names, argument meanings and errors follow the reference's functions
(paths within the reference project):

- ``spmv`` / ``spmm`` with ``Product``: compute/product/mod.rs:31-110;
- ``pagerank`` with ``PageRank`` -> ``Ranks``: compute/pagerank/mod.rs:27-151;
- ``bfs`` / ``reachable_set`` / ``reachable`` with ``Limits`` ->
  ``Traversed``: traversal/bfs.rs:14-60, reachable.rs:18-90, limits.rs,
  stats.rs;
- ``eigen`` with ``EigenOptions`` -> ``Eigen``: spectral/lanczos.rs:136-224;
- ``top_k``: compute/ranking.rs:52.

Operands are numpy arrays (host) or torch CUDA tensors (device); the
library tells them apart.  Errors raise the ``ComputeError`` /
``TraversalError`` / ``SpectralError`` subclasses named as the reference's
variants.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

from . import _abi as A

# ----------------------------------------------------------------- errors


class WarrenError(Exception):
    """A non-OK wc_status, with the library's detail."""

    def __init__(self, status: int, detail: Optional[A.ErrorDetail] = None):
        self.status = status
        self.detail = detail
        msg = A.load().wc_status_name(status).decode()
        if detail is not None and detail.message:
            msg = f"{msg}: {detail.message.decode(errors='replace')}"
        super().__init__(msg)


class ComputeError(WarrenError):
    pass


class MemoryLimit(ComputeError):
    pass


class OutOfMemory(ComputeError):
    pass


class DtypeMismatch(ComputeError):
    pass


class IdSpaceMismatch(ComputeError):
    pass


class WidthMismatch(ComputeError):
    pass


class UnknownSemiring(ComputeError):
    pass


class UnknownBinaryOp(ComputeError):
    pass


class ZeroWidth(ComputeError):
    pass


class Cancelled(ComputeError):
    pass


class ArithmeticError_(ComputeError):
    """ComputeError::Arithmetic (compute/error.rs:150-152)."""


class BigintOutOfRange(ArithmeticError_):
    pass


class FloatOverflow(ArithmeticError_):
    pass


class FloatUnderflow(ArithmeticError_):
    pass


class DivisionByZero(ArithmeticError_):
    pass


class TraversalError(WarrenError):
    pass


class NodeOutsideIdSpace(TraversalError):
    pass


class NodeFilterIdSpace(TraversalError):
    pass


class ReverseCsrMissing(TraversalError):
    pass


class SpectralError(WarrenError):
    pass


class NotSymmetric(SpectralError):
    pass


class NonPositiveDegree(SpectralError):
    pass


class EigenpairCount(SpectralError):
    pass


class WorkingSet(SpectralError):
    pass


class NotFinite(SpectralError):
    pass


class GraphError(WarrenError):
    """graph/error.rs: a stored segment or CSR that does not decode."""


class SegmentTruncated(GraphError):
    pass


class SegmentMagic(GraphError):
    pass


class SegmentFormat(GraphError):
    pass


class SegmentKind(GraphError):
    pass


class SegmentReserved(GraphError):
    pass


class SegmentWidth(GraphError):
    pass


class SegmentLength(GraphError):
    pass


class OffsetsLength(GraphError):
    pass


class FirstOffsetNotZero(GraphError):
    pass


class StoredRowsNotAscending(GraphError):
    pass


class StoredRowOutsideIdSpace(GraphError):
    pass


class StoredRowEmpty(GraphError):
    pass


class OffsetsNotMonotone(GraphError):
    pass


class FinalOffset(GraphError):
    pass


class TargetOutsideIdSpace(GraphError):
    pass


class RowNotSorted(GraphError):
    pass


class WeightsLength(GraphError):
    pass


class BackendError(WarrenError):
    pass


class InvalidArgument(BackendError):
    pass


class Unsupported(BackendError):
    pass


class CudaError(BackendError):
    pass


class DeviceTimeout(BackendError):
    pass


class NoDevice(BackendError):
    pass


_ERRORS = {
    1: MemoryLimit, 2: OutOfMemory, 3: DtypeMismatch, 4: IdSpaceMismatch, 5: WidthMismatch,
    6: UnknownSemiring, 7: UnknownBinaryOp, 8: ZeroWidth, 9: Cancelled, 10: BigintOutOfRange,
    11: FloatOverflow, 12: FloatUnderflow, 13: DivisionByZero, 20: NodeOutsideIdSpace,
    21: NodeFilterIdSpace, 22: ReverseCsrMissing, 30: NotSymmetric, 31: NonPositiveDegree,
    32: EigenpairCount, 33: WorkingSet, 34: NotFinite, 40: InvalidArgument, 41: Unsupported,
    42: CudaError, 43: DeviceTimeout, 44: NoDevice,
    50: SegmentTruncated, 51: SegmentMagic, 52: SegmentFormat, 53: SegmentKind,
    54: SegmentReserved, 55: SegmentWidth, 56: SegmentLength, 57: OffsetsLength,
    58: FirstOffsetNotZero, 59: StoredRowsNotAscending, 60: StoredRowOutsideIdSpace,
    61: StoredRowEmpty, 62: OffsetsNotMonotone, 63: FinalOffset, 64: TargetOutsideIdSpace,
    65: RowNotSorted, 66: WeightsLength,
}


def _raise(status: int, detail: A.ErrorDetail):
    if status != 0:
        raise _ERRORS.get(status, WarrenError)(status, detail)


# ----------------------------------------------------------------- operands

_DTYPES = {np.dtype(np.float64): A.F64, np.dtype(np.float32): A.F32, np.dtype(np.int64): A.I64,
           np.dtype(np.uint8): A.BOOL, np.dtype(np.bool_): A.BOOL}
_TORCH_DTYPES = {"torch.float64": A.F64, "torch.float32": A.F32, "torch.int64": A.I64,
                 "torch.uint8": A.BOOL, "torch.bool": A.BOOL}


def _ptr(a) -> Optional[int]:
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        if not a.flags["C_CONTIGUOUS"]:
            raise ValueError("operands must be C-contiguous")
        return a.ctypes.data
    if hasattr(a, "data_ptr"):
        if not a.is_contiguous():
            raise ValueError("operands must be contiguous")
        return a.data_ptr()
    raise TypeError(f"unsupported operand {type(a)}")


def _dtype(a) -> int:
    if isinstance(a, np.ndarray):
        return _DTYPES[a.dtype]
    return _TORCH_DTYPES[str(a.dtype)]


def _len(a) -> int:
    return a.shape[0] if len(a.shape) else 1


# ----------------------------------------------------------------- runtime


class Budget:
    """compute/memory.rs (ComputeMemory): device bytes charged before use."""

    def __init__(self, limit: int = 1 << 62):
        h = A.P()
        _raise(A.load().wc_budget_create(limit, C.byref(h)), A.ErrorDetail())
        self.handle = h
        self.limit = limit

    @property
    def in_use(self) -> int:
        return A.load().wc_budget_in_use(self.handle)

    @property
    def peak(self) -> int:
        return A.load().wc_budget_peak(self.handle)

    def __del__(self):
        h = getattr(self, "handle", None)
        if h:
            try:
                A.load().wc_budget_destroy(h)
            except Exception:  # interpreter shutdown
                pass
            self.handle = None


class Interrupts:
    """A host cancel word and a progress hook (interrupts.rs, progress.rs)."""

    def __init__(self, progress=None):
        self.word = C.c_int32(0)
        self.progress = progress
        self.phases: list = []

    def cancel(self):
        self.word.value = 1


def _call(interrupts: Optional[Interrupts] = None, stream=None, flags: int = 0,
          memory: Optional[Budget] = None):
    detail = A.ErrorDetail()
    call = A.Call()
    call.detail = C.pointer(detail)
    if memory is not None:
        call.memory = memory.handle
    if interrupts is not None:
        call.cancel = C.pointer(interrupts.word)
        if interrupts.progress is not None:
            cb = A.PROGRESS_FN(lambda ctx, phase, done, total: interrupts.progress(
                phase.decode(), done, None if total == 2**64 - 1 else total))
            call.progress = cb
            call._keep = cb  # noqa: keep the callback alive for the call
    if stream is not None:
        call.stream = stream if isinstance(stream, int) else getattr(stream, "cuda_stream", None)
    call.flags = flags
    return call, detail


CALL_ASYNC = 1
CALL_TIMING = 2


class GraphVersion:
    """A version's device copy: the CSR and reverse CSR of a built version
    (graph/csr/mod.rs:38-237), keyed by (graph, version)."""

    def __init__(self, offsets, targets, weights=None, reverse=True, budget: Budget = None,
                 graph_id: int = 0, version: int = 0):
        offsets = np.ascontiguousarray(offsets, dtype=np.uint64)
        targets = np.ascontiguousarray(targets, dtype=np.uint32)
        n = len(offsets) - 1
        m = len(targets)
        csr = A.CsrHost(n, m, offsets.ctypes.data, targets.ctypes.data, None, None, None, None,
                        0)
        self._keep = [offsets, targets]
        if weights is not None:
            weights = np.ascontiguousarray(weights, dtype=np.float64)
            csr.weights = weights.ctypes.data
            self._keep.append(weights)
        if reverse is True:
            # The version has a reverse CSR: the library transposes on the device.
            csr.reverse_on_device = 1
        elif reverse:
            roff, rtgt, rw = reverse
            roff = np.ascontiguousarray(roff, dtype=np.uint64)
            rtgt = np.ascontiguousarray(rtgt, dtype=np.uint32)
            rw = None if rw is None else np.ascontiguousarray(rw, dtype=np.float64)
            csr.reverse_offsets, csr.reverse_targets = roff.ctypes.data, rtgt.ctypes.data
            csr.reverse_weights = _ptr(rw)
            self._keep += [roff, rtgt, rw]
        self.budget = budget or Budget()
        call, detail = _call()
        h = A.P()
        _raise(A.load().wc_version_upload(graph_id, version, C.byref(csr), self.budget.handle,
                                          C.byref(call), C.byref(h)), detail)
        self._keep = None
        self.handle = h
        self.id_space = n
        self.edges = m
        self.weighted = weights is not None

    @classmethod
    def from_segments(cls, id_space: int, offsets: bytes, targets: bytes, weights=None,
                      rows=None, reverse: bool = True, budget: Budget = None,
                      graph_id: int = 0, version: int = 0) -> "GraphVersion":
        """A version loaded straight from its stored CSR segments
        (graph/segment/csr.rs:83-122), checked on the device as the
        reference's decode checks them."""
        self = cls.__new__(cls)
        self.budget = budget or Budget()
        bufs = [None if b is None else np.frombuffer(bytes(b), np.uint8)
                for b in (rows, offsets, targets, weights)]
        # An empty segment is passed as a non-null pointer to no bytes.
        ptr = [None if b is None else (b.ctypes.data if len(b) else 1) for b in bufs]
        ln = [0 if b is None else len(b) for b in bufs]
        call, detail = _call()
        h = A.P()
        _raise(A.load().wc_version_load_segments(
            graph_id, version, id_space, ptr[0], ln[0], ptr[1], ln[1], ptr[2], ln[2], ptr[3],
            ln[3], int(bool(reverse)), self.budget.handle, C.byref(call), C.byref(h)), detail)
        self.handle = h
        info = self.info()
        self.id_space, self.edges, self.weighted = info.id_space, info.edges, bool(info.weighted)
        return self

    def info(self) -> A.VersionInfo:
        info = A.VersionInfo()
        _raise(A.load().wc_version_info_get(self.handle, C.byref(info)), A.ErrorDetail())
        return info

    def sync(self, interrupts=None):
        call, detail = _call(interrupts)
        _raise(A.load().wc_version_sync(self.handle, C.byref(call)), detail)

    def release(self):
        """Frees the device copy; refused (InvalidArgument) while a cursor
        over it is open."""
        h = getattr(self, "handle", None)
        if h:
            _raise(A.load().wc_version_release(h), A.ErrorDetail())
            self.handle = None

    def __del__(self):
        try:
            self.release()
        except Exception:  # interpreter shutdown: the library is already gone
            pass

    def timing(self, phase: str):
        """(device ms, kernels launched) of kernel group `phase` ("level",
        "depth", "iteration") in the last call made with timing=True."""
        n = C.c_uint32(0)
        ms = A.load().wc_version_timing(self.handle, phase.encode(), C.byref(n))
        return ms, n.value


def host_reverse(offsets, targets, weights=None):
    """The reverse CSR by the host's counting transpose
    (graph/csr/transpose.rs:14-44): (offsets, targets, weights or None), to
    give GraphVersion(reverse=...) instead of the device transpose."""
    offsets = np.ascontiguousarray(offsets, dtype=np.uint64)
    targets = np.ascontiguousarray(targets, dtype=np.uint32)
    n, m = len(offsets) - 1, len(targets)
    roff = np.zeros(n + 1, np.uint64)
    rtgt = np.zeros(max(m, 1), np.uint32)
    rw = None
    if weights is not None:
        weights = np.ascontiguousarray(weights, dtype=np.float64)
        rw = np.zeros(max(m, 1), np.float64)
    _raise(A.load().wc_host_transpose(n, m, offsets.ctypes.data, targets.ctypes.data,
                                      _ptr(weights), roff.ctypes.data, rtgt.ctypes.data,
                                      _ptr(rw)), A.ErrorDetail())
    return roff, rtgt[:m], None if rw is None else rw[:m]


def encode_segment(kind: int, elements: np.ndarray) -> bytes:
    """One stored segment as the reference writes it (graph/segment/mod.rs:
    1-16, 190-272): the 16-byte header (magic, format 2 for a CSR's
    segments, kind, element width, reserved 0, count) and the little-endian
    elements.  Kinds: offsets 1, targets 2, weights 3, rows 11."""
    elements = np.ascontiguousarray(elements)
    header = b"WRSG" + bytes([2, kind, elements.dtype.itemsize, 0])
    return header + int(len(elements)).to_bytes(8, "little") + elements.astype(
        elements.dtype.newbyteorder("<"), copy=False).tobytes()


def csr_segments(offsets, targets, weights=None, sparse: bool = False):
    """A CSR's segments (segment/csr.rs:124-131): (rows or None, offsets,
    targets, weights or None); with `sparse`, only the non-empty rows are
    stored, with one offset each plus the end."""
    offsets = np.asarray(offsets, np.uint64)
    rows = None
    if sparse:
        keep = np.nonzero(np.diff(offsets))[0]
        rows = encode_segment(11, keep.astype(np.uint32))
        offsets = np.append(offsets[keep], offsets[-1]).astype(np.uint64)
    return (rows, encode_segment(1, offsets), encode_segment(2, np.asarray(targets, np.uint32)),
            None if weights is None else encode_segment(3, np.asarray(weights, np.float64)))


# ----------------------------------------------------------------- products


@dataclass
class Product:
    """compute/product/mod.rs:31-56."""

    semiring: str = "plus_times"
    transpose: bool = False
    weighted: Optional[bool] = None
    mask: object = None
    complement: bool = False
    replace: bool = False
    accumulate: Optional[str] = None


def _product_c(p: Product):
    name = {"or_and": "lor_land"}.get(p.semiring, p.semiring)
    if name not in A.SEMIRINGS:
        raise UnknownSemiring(6)
    acc = A.OP_NONE
    if p.accumulate is not None:
        if p.accumulate not in A.BINARY_OPS:
            raise UnknownBinaryOp(7)
        acc = A.BINARY_OPS.index(p.accumulate)
    pc = A.ProductC(A.SEMIRINGS.index(name), int(p.transpose),
                    -1 if p.weighted is None else int(p.weighted), None, int(p.replace), acc)
    mask = None
    if p.mask is not None:
        mask = A.Mask(_ptr(p.mask), _dtype(p.mask), int(p.complement))
        pc.mask = C.pointer(mask)
    return pc, mask


def _check_operands(graph: GraphVersion, x, y, width: Optional[int]):
    if _dtype(x) != _dtype(y):
        raise DtypeMismatch(3)
    for v in (x, y):
        if _len(v) != graph.id_space:
            raise IdSpaceMismatch(4)
    wx = 1 if len(x.shape) == 1 else x.shape[1]
    wy = 1 if len(y.shape) == 1 else y.shape[1]
    if width == 1 and (wx != 1 or wy != 1):
        raise WidthMismatch(5)
    if wx != wy:
        raise WidthMismatch(5)
    return wx


def spmv(graph: GraphVersion, product: Product, x, y, interrupts=None, stream=None,
         asynchronous=False, memory: Optional[Budget] = None):
    """y = A ⊗ x (or Aᵀ ⊗ x), y updated in place (product/mod.rs:77-92).
    `memory`: the call's own budget (ComputeMemory) for its working memory."""
    _check_operands(graph, x, y, 1)
    pc, mask = _product_c(product)
    call, detail = _call(interrupts, stream, 1 if asynchronous else 0, memory)
    _raise(A.load().wc_spmv(graph.handle, C.byref(call), C.byref(pc), _dtype(y), _ptr(x), _ptr(y)),
           detail)


def spmm(graph: GraphVersion, product: Product, x, y, interrupts=None, stream=None,
         memory: Optional[Budget] = None):
    """Y = A ⊗ X over row-major id_space × width matrices (product/mod.rs:97-110)."""
    width = _check_operands(graph, x, y, None)
    pc, mask = _product_c(product)
    call, detail = _call(interrupts, stream, 0, memory)
    _raise(A.load().wc_spmm(graph.handle, C.byref(call), C.byref(pc), _dtype(y), width, _ptr(x),
                            _ptr(y)), detail)


# ----------------------------------------------------------------- pagerank


@dataclass
class PageRank:
    """compute/pagerank/mod.rs:27-47 (all relations)."""

    damping: float = 0.85
    tol: Optional[float] = 1e-6
    max_iter: int = 100
    weighted: Optional[bool] = None
    seed: object = None


@dataclass
class Ranks:
    values: object
    iterations: int


def _pr_opts(p: PageRank):
    seed = None
    if p.seed is not None:
        seed = p.seed if not isinstance(p.seed, np.ndarray) else np.ascontiguousarray(
            p.seed, dtype=np.float64)
        if isinstance(seed, np.ndarray) and seed.dtype == np.bool_:
            raise DtypeMismatch(3)
    o = A.PageRankOpts(p.damping, 0.0 if p.tol is None else p.tol, int(p.tol is not None),
                       -1 if p.weighted is None else int(p.weighted), p.max_iter, _ptr(seed))
    return o, seed


def pagerank(graph: GraphVersion, tombstones=None, pagerank: PageRank = PageRank(), out=None,
             interrupts=None, stream=None, timing=False, memory: Optional[Budget] = None,
             timeout_ms: int = 0) -> Ranks:
    """compute/pagerank/mod.rs:96-151; `tombstones` are NodeSet words.
    `memory`: the call's own budget; `timeout_ms`: a bound on the wait for
    the device (0: the library's default), past which the call stops its
    kernels and raises DeviceTimeout."""
    o, seed = _pr_opts(pagerank)
    ranks = out if out is not None else np.zeros(graph.id_space, np.float64)
    it = C.c_uint32(0)
    call, detail = _call(interrupts, stream, CALL_TIMING if timing else 0, memory)
    call.timeout_ms = timeout_ms
    _raise(A.load().wc_pagerank(graph.handle, C.byref(call), C.byref(o), _ptr(tombstones),
                                _ptr(ranks), C.byref(it)), detail)
    return Ranks(ranks, it.value)


def pagerank_noalloc(graph: GraphVersion, tombstones=None, pagerank: PageRank = PageRank(),
                     out=None, interrupts=None, stream=None) -> Ranks:
    """pagerank() through wc_pagerank_noalloc: no allocation inside the call;
    the working memory is the library's fixed 64 MiB device array."""
    o, seed = _pr_opts(pagerank)
    ranks = out if out is not None else np.zeros(graph.id_space, np.float64)
    it = C.c_uint32(0)
    call, detail = _call(interrupts, stream)
    _raise(A.load().wc_pagerank_noalloc(graph.handle, C.byref(call), C.byref(o),
                                        _ptr(tombstones), _ptr(ranks), C.byref(it)), detail)
    return Ranks(ranks, it.value)


def random_uniform(graph: GraphVersion, seed: int, stream: int = 0, out=None):
    """compute/random.rs:11-25 evaluated on the device over the version's id
    space (the start vectors wc_eigen draws)."""
    x = out if out is not None else np.zeros(graph.id_space, np.float64)
    call, detail = _call()
    _raise(A.load().wc_random_uniform(graph.handle, C.byref(call), seed, stream, _ptr(x)), detail)
    return x


def selftest_bounded_wait(limit_us: int, stream=None):
    """A device wait that nothing completes, bounded to `limit_us`: raises
    DeviceTimeout once it gives up (wc_selftest_bounded_wait)."""
    call, detail = _call(None, stream)
    _raise(A.load().wc_selftest_bounded_wait(C.byref(call), limit_us), detail)


def last_margin(graph: GraphVersion) -> float:
    return A.load().wc_pagerank_last_margin(graph.handle)


def node_set(id_space: int, ids) -> np.ndarray:
    """NodeSet bitmap words (traversal/node_set.rs, graph/tombstones.rs)."""
    words = np.zeros((id_space + 63) // 64, np.uint64)
    ids = np.asarray(list(ids), dtype=np.uint64)
    if len(ids):
        np.bitwise_or.at(words, (ids // 64).astype(np.int64),
                         np.left_shift(np.uint64(1), ids % np.uint64(64)))
    return words


# ----------------------------------------------------------------- traversal


@dataclass
class Limits:
    """traversal/limits.rs:4-12."""

    max_depth: Optional[int] = None
    max_results: Optional[int] = None


@dataclass
class Visit:
    node: int
    depth: int
    via: Optional[int]


@dataclass
class TraversalStats:
    nodes_visited: int = 0
    edges_traversed: int = 0
    truncated: bool = False
    levels: int = 0
    pulled_levels: int = 0


@dataclass
class Traversed:
    result: object
    stats: TraversalStats


_DIRECTIONS = {"out": A.OUT, "in": A.IN, "both": A.BOTH}


def _stats(s: A.TraversalStats) -> TraversalStats:
    return TraversalStats(s.nodes_visited, s.edges_traversed, bool(s.truncated), s.levels,
                          s.pulled_levels)


def _limits(limits: Limits) -> A.Limits:
    return A.Limits(A.UNREACHED if limits.max_depth is None else limits.max_depth,
                    2**64 - 1 if limits.max_results is None else limits.max_results)


def bfs(graph: GraphVersion, starts: Sequence[int], filter=None, limits: Limits = Limits(),
        direction: str = "out", interrupts=None) -> Traversed:
    """traversal/bfs.rs:34-45: every node reached, once, in BFS order."""
    st = np.ascontiguousarray(np.asarray(starts, dtype=np.uint64))
    filt = None
    if filter is not None:
        filt = node_set(graph.id_space, filter) if not isinstance(filter, np.ndarray) else filter
    rows = np.zeros(3 * (graph.id_space + 1), np.uint64)
    count = C.c_uint64(0)
    stats = A.TraversalStats()
    lim = _limits(limits)
    call, detail = _call(interrupts)
    _raise(A.load().wc_bfs_visits(graph.handle, C.byref(call), _DIRECTIONS[direction], _ptr(st),
                                  len(st), C.byref(lim), _ptr(filt), _ptr(rows),
                                  graph.id_space + 1, C.byref(count), C.byref(stats)), detail)
    r = rows[: 3 * count.value].reshape(-1, 3)
    visits = [Visit(int(a), int(b), None if int(c) == A.NO_VIA else int(c)) for a, b, c in r]
    return Traversed(visits, _stats(stats))


def bfs_depths(graph: GraphVersion, starts, max_depth=None, direction="out", filter=None,
               depth_out=None, via_out=None):
    """The per-node form of bfs: (depth u32[n], via u64[n], stats)."""
    st = np.ascontiguousarray(np.asarray(starts, dtype=np.uint64))
    d = depth_out if depth_out is not None else np.zeros(graph.id_space, np.uint32)
    v = via_out if via_out is not None else np.zeros(graph.id_space, np.uint64)
    stats = A.TraversalStats()
    lim = _limits(Limits(max_depth, None))
    call, detail = _call()
    _raise(A.load().wc_bfs(graph.handle, C.byref(call), _DIRECTIONS[direction], _ptr(st), len(st),
                           C.byref(lim), _ptr(filter), _ptr(d), _ptr(v), C.byref(stats)), detail)
    return d, v, _stats(stats)


def reachable_set(graph: GraphVersion, starts, max_depth=None, direction="out",
                  interrupts=None) -> Traversed:
    """traversal/reachable.rs:48-58."""
    st = np.ascontiguousarray(np.asarray(starts, dtype=np.uint64))
    nodes = np.zeros(graph.id_space + 1, np.uint64)
    count = C.c_uint64(0)
    stats = A.TraversalStats()
    call, detail = _call(interrupts)
    _raise(A.load().wc_reachable_set(graph.handle, C.byref(call), _DIRECTIONS[direction], _ptr(st),
                                     len(st), A.UNREACHED if max_depth is None else max_depth,
                                     _ptr(nodes), len(nodes), C.byref(count), C.byref(stats)),
           detail)
    return Traversed([int(v) for v in nodes[: count.value]], _stats(stats))


class BfsCursor:
    """traversal/bfs_cursor.rs:17-138: bfs (or, with `reachable=True`,
    reachable_set) run one level per next_level call.  The cursor keeps
    its graph alive and its own device buffers until close()."""

    def __init__(self, graph: GraphVersion, starts, filter=None, limits: Limits = Limits(),
                 direction: str = "out", reachable: bool = False, interrupts=None):
        st = np.ascontiguousarray(np.asarray(starts, dtype=np.uint64))
        filt = None
        if filter is not None:
            filt = node_set(graph.id_space, filter) if not isinstance(filter, np.ndarray) \
                else filter
        lim = _limits(limits)
        call, detail = _call(interrupts)
        handle = C.c_void_p()
        _raise(A.load().wc_bfs_cursor_open(graph.handle, C.byref(call), _DIRECTIONS[direction],
                                           _ptr(st), len(st), C.byref(lim), _ptr(filt),
                                           1 if reachable else 0, C.byref(handle)), detail)
        self.graph = graph
        self.handle = handle.value

    @classmethod
    def reachable_set(cls, graph: GraphVersion, starts, max_depth=None, direction="out",
                      interrupts=None) -> "BfsCursor":
        """bfs_cursor.rs:75-88."""
        return cls(graph, starts, None, Limits(max_depth, None), direction, True, interrupts)

    def next_level(self, visitor=None, interrupts=None):
        """bfs_cursor.rs:90-126: runs the next level and hands its visits
        to `visitor` (a callable; a true return breaks, as
        ControlFlow::Break) or returns them when no visitor is given.
        Returns (visits, more) without a visitor, else `more`."""
        if self.handle is None:
            raise ValueError("cursor closed")
        call, detail = _call(interrupts)
        count = C.c_uint64(0)
        more = C.c_int32(0)
        lib = A.load()
        _raise(lib.wc_bfs_cursor_next(self.handle, C.byref(call), C.byref(count),
                                      C.byref(more)), detail)
        rows = np.zeros((count.value, 3), np.uint64)
        if count.value:
            _raise(lib.wc_bfs_cursor_read(self.handle, 0, count.value, _ptr(rows)), detail)
        visits = [Visit(int(a), int(b), None if int(c) == A.NO_VIA else int(c)) for a, b, c in rows]
        if visitor is None:
            return visits, bool(more.value)
        for i, visit in enumerate(visits):
            if visitor(visit):
                _raise(lib.wc_bfs_cursor_stop(self.handle, C.byref(call), i + 1), detail)
                return False
        return bool(more.value)

    def stats(self) -> TraversalStats:
        stats = A.TraversalStats()
        _raise(A.load().wc_bfs_cursor_stats(self.handle, C.byref(stats)), A.ErrorDetail())
        return _stats(stats)

    def close(self):
        if self.handle is not None:
            A.load().wc_bfs_cursor_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def components(graph: GraphVersion, labels_out=None, interrupts=None):
    """traversal/components.rs:21-58: each dense id's weakly connected
    component, labelled by its smallest dense id: (labels u64[n], stats)."""
    labels = labels_out if labels_out is not None else np.zeros(graph.id_space, np.uint64)
    stats = A.TraversalStats()
    call, detail = _call(interrupts)
    _raise(A.load().wc_components(graph.handle, C.byref(call), _ptr(labels), C.byref(stats)),
           detail)
    return labels, _stats(stats)


# --------------------------------------------------------------- vector map

_MAP_NP = {"f32": np.float32, "f64": np.float64, "i64": np.int64, "bool": np.bool_}


class UnknownOperand(ComputeError):
    pass


class OperandType(ComputeError):
    pass


class NullResult(ComputeError):
    pass


class SqrtOfNegative(ArithmeticError_):
    pass


class LogOfZero(ArithmeticError_):
    pass


class LogOfNegative(ArithmeticError_):
    pass


class ZeroToNegativePower(ArithmeticError_):
    pass


class ComplexPower(ArithmeticError_):
    pass


_ERRORS.update({14: SqrtOfNegative, 15: LogOfZero, 16: LogOfNegative, 17: ZeroToNegativePower,
                18: ComplexPower, 70: UnknownOperand, 71: OperandType, 72: NullResult})


def vector_map(graph: GraphVersion, expr, operands=(), out=None, interrupts=None):
    """compute/map/mod.rs:49-78 (map): `expr` (a pg_warren_b200.expr tree)
    at every element of the version's id space, over `operands` (numpy
    arrays or CUDA tensors, id_space rows, width 1 or the widest width);
    returns the result, id_space × width of the expression's type."""
    from . import expr as X
    nodes, children, root = X.serialize(expr)
    ops = [np.ascontiguousarray(o) if isinstance(o, np.ndarray) else o for o in operands]
    count = len(ops)
    ptrs = (C.c_void_p * max(count, 1))(*[_ptr(o) for o in ops])
    dtypes = (C.c_int32 * max(count, 1))(*[_dtype(o) for o in ops])
    spaces = (C.c_uint64 * max(count, 1))(*[_len(o) for o in ops])
    widths = (C.c_uint32 * max(count, 1))(*[1 if len(o.shape) == 1 else int(o.shape[1])
                                            for o in ops])
    width = max([1] + list(widths[:count]))
    if out is None:
        shape = (graph.id_space,) if width == 1 else (graph.id_space, width)
        out = np.zeros(shape, _MAP_NP[expr.type])
    got = C.c_uint32(0)
    call, detail = _call(interrupts)
    _raise(A.load().wc_vector_map(graph.handle, C.byref(call), nodes.ctypes.data, len(nodes),
                                  children.ctypes.data if len(children) else None, len(children),
                                  root, ptrs, dtypes, spaces, widths, count, _ptr(out),
                                  C.byref(got)), detail)
    return out


# ------------------------------------------------------------ vector reduce

REDUCTIONS = ["sum", "max", "min", "l1", "l2", "nnz"]  # compute/reduce.rs:23-38
NORMS = ["l1", "l2", "linf"]                            # compute/reduce.rs:74-82


def _reduction(name: str, names) -> int:
    if name not in names:
        raise InvalidArgument(40)  # reduce.rs:64-72: an unknown reduction or norm
    return names.index(name)


def vector_reduce(graph: GraphVersion, x, reduction: str, tombstones=None, interrupts=None):
    """compute/reduce.rs:118-153 (reduce, or reduce_live with tombstones):
    `reduction` over x's id_space × width elements; None for the max or
    min of no elements."""
    width = 1 if getattr(x, "ndim", 1) == 1 else int(x.shape[1])
    if _len(x) != graph.id_space:
        raise IdSpaceMismatch(4)
    out = C.c_double(0.0)
    null = C.c_int32(0)
    call, detail = _call(interrupts)
    _raise(A.load().wc_vector_reduce(graph.handle, C.byref(call), _dtype(x), _ptr(x), width,
                                     _ptr(tombstones), _reduction(reduction, REDUCTIONS),
                                     C.byref(out), C.byref(null)), detail)
    return None if null.value else out.value


def vector_norm_diff(graph: GraphVersion, a, b, norm: str, interrupts=None) -> float:
    """compute/reduce.rs:175-206 (norm_diff): norm(a - b), a row past the
    shorter vector's end counting as zero."""
    wa = 1 if getattr(a, "ndim", 1) == 1 else int(a.shape[1])
    wb = 1 if getattr(b, "ndim", 1) == 1 else int(b.shape[1])
    if wa != wb:
        raise WidthMismatch(5)
    out = C.c_double(0.0)
    call, detail = _call(interrupts)
    _raise(A.load().wc_vector_norm_diff(graph.handle, C.byref(call), _dtype(a), _ptr(a), _len(a),
                                        _dtype(b), _ptr(b), _len(b), wa,
                                        _reduction(norm, NORMS), C.byref(out)), detail)
    return out.value


# -------------------------------------------------------------- centrality


@dataclass
class Sampling:
    """compute/centrality/sources.rs:22-33: `k` sources drawn with `seed`
    from the live nodes `population` (a per-node mask, nonzero selects;
    None: every node) selects; k None takes them all."""

    k: Optional[int] = None
    seed: int = 0
    population: Optional[np.ndarray] = None
    complement: bool = False


@dataclass
class Centrality:
    """compute/centrality/mod.rs:67-73: the values and the number of sources."""

    values: np.ndarray
    sources: int


def sample_sources(id_space: int, sampling: Sampling = Sampling(), tombstones=None) -> np.ndarray:
    """The sources `sampling` chooses among the live nodes, ascending
    (Sources::choose, sources.rs:55-95)."""
    pop = None
    if sampling.population is not None:
        pop = np.ascontiguousarray(np.asarray(sampling.population) != 0, dtype=np.uint8)
        if len(pop) != id_space:
            raise IdSpaceMismatch(4)
    out = np.zeros(max(id_space, 1), np.uint64)
    count = C.c_uint64(0)
    k = -1 if sampling.k is None else int(sampling.k)
    _raise(A.load().wc_sample_sources(id_space, _ptr(tombstones), _ptr(pop),
                                      int(sampling.complement), k, sampling.seed & (2**64 - 1),
                                      _ptr(out), C.byref(count)), A.ErrorDetail())
    return out[:count.value].copy()


def _centrality(graph: GraphVersion, measure: int, sampling: Sampling, tombstones,
                wf_improved: bool, columns_per_pass: int, interrupts, sources) -> Centrality:
    if sources is None:
        sources = sample_sources(graph.id_space, sampling, tombstones)
    sources = np.ascontiguousarray(sources, dtype=np.uint64)
    values = np.zeros(graph.id_space, np.float64)
    o = A.CentralityOpts(measure, int(wf_improved), columns_per_pass, 0)
    call, detail = _call(interrupts)
    _raise(A.load().wc_centrality(graph.handle, C.byref(call), C.byref(o), _ptr(sources),
                                  len(sources), _ptr(tombstones), _ptr(values)), detail)
    return Centrality(values, len(sources))


def closeness_centrality(graph: GraphVersion, sampling: Sampling = Sampling(),
                         wf_improved: bool = True, tombstones=None, columns_per_pass: int = 0,
                         interrupts=None, sources=None) -> Centrality:
    """compute/centrality/closeness.rs:36-45 on the version's unweighted
    forward rows (an undirected graph: upload it symmetrised).  `sources`
    (ascending, as sample_sources gives them) replaces the sampling."""
    return _centrality(graph, 0, sampling, tombstones, wf_improved, columns_per_pass, interrupts,
                       sources)


def harmonic_centrality(graph: GraphVersion, sampling: Sampling = Sampling(), tombstones=None,
                        columns_per_pass: int = 0, interrupts=None, sources=None) -> Centrality:
    """compute/centrality/closeness.rs:49-56, as closeness_centrality."""
    return _centrality(graph, 1, sampling, tombstones, False, columns_per_pass, interrupts,
                       sources)


def betweenness_centrality(graph: GraphVersion, sampling: Sampling = Sampling(),
                           normalized: bool = True, endpoints: bool = False,
                           directed: bool = True, tombstones=None, interrupts=None,
                           sources=None) -> Centrality:
    """compute/centrality/betweenness.rs:27-38 on the version's unweighted
    forward rows (an undirected graph: upload it symmetrised and pass
    directed=False, which the rescale reads)."""
    if sources is None:
        sources = sample_sources(graph.id_space, sampling, tombstones)
    sources = np.ascontiguousarray(sources, dtype=np.uint64)
    values = np.zeros(graph.id_space, np.float64)
    o = A.BetweennessOpts(int(normalized), int(endpoints), int(directed), 0)
    call, detail = _call(interrupts)
    _raise(A.load().wc_betweenness(graph.handle, C.byref(call), C.byref(o), _ptr(sources),
                                   len(sources), _ptr(tombstones), _ptr(values)), detail)
    return Centrality(values, len(sources))


def reachable(graph: GraphVersion, start: int, target: int, max_depth=None,
              direction="out") -> Traversed:
    """traversal/reachable.rs:18-43."""
    r = C.c_int32(0)
    stats = A.TraversalStats()
    call, detail = _call()
    _raise(A.load().wc_reachable(graph.handle, C.byref(call), _DIRECTIONS[direction], start,
                                 target, A.UNREACHED if max_depth is None else max_depth,
                                 C.byref(r), C.byref(stats)), detail)
    return Traversed(bool(r.value), _stats(stats))


# ----------------------------------------------------------------- batched


def bfs_batched(graph: GraphVersion, sources, max_depths, depth_out=None, edges_out=None,
                stream=None, timing=False, interrupts=None, memory: Optional[Budget] = None,
                timeout_ms: int = 0):
    """`len(sources)` BFS searches as one bit-packed boolean SpMM: depths
    u8[k, n] (255: not reached within the source's cap).  Sources, caps and
    outputs may be host arrays or device tensors."""
    src = sources if hasattr(sources, "data_ptr") else np.ascontiguousarray(
        np.asarray(sources, dtype=np.uint64))
    caps = max_depths if hasattr(max_depths, "data_ptr") else np.ascontiguousarray(
        np.asarray(max_depths, dtype=np.uint32))
    k = len(src)
    d = depth_out if depth_out is not None else np.zeros((k, graph.id_space), np.uint8)
    e = edges_out if edges_out is not None else np.zeros(k, np.uint64)
    call, detail = _call(interrupts, stream, CALL_TIMING if timing else 0, memory)
    call.timeout_ms = timeout_ms
    _raise(A.load().wc_bfs_batched(graph.handle, C.byref(call), _ptr(src), _ptr(caps), k, _ptr(d),
                                   _ptr(e)), detail)
    return d, e


def minplus_batched(graph: GraphVersion, sources, max_hops, dist_out=None, iterations_out=None):
    """`len(sources)` hop-bounded min-plus searches (the sssp_vector loop)."""
    src = np.ascontiguousarray(np.asarray(sources, dtype=np.uint64))
    hops = np.ascontiguousarray(np.asarray(max_hops, dtype=np.uint32))
    k = len(src)
    d = dist_out if dist_out is not None else np.zeros((k, graph.id_space), np.int64)
    it = iterations_out if iterations_out is not None else np.zeros(k, np.uint32)
    call, detail = _call()
    _raise(A.load().wc_minplus_batched(graph.handle, C.byref(call), _ptr(src), _ptr(hops), k,
                                       _ptr(d), _ptr(it)), detail)
    return d, it


def ppr_batched(graph: GraphVersion, seed_sets, pagerank: PageRank = PageRank(), ranks_out=None,
                iterations_out=None):
    """Personalised PageRank per seed set, each column stopping on its own."""
    offs = np.zeros(len(seed_sets) + 1, np.uint64)
    for i, s in enumerate(seed_sets):
        offs[i + 1] = offs[i] + len(s)
    nodes = np.ascontiguousarray(np.concatenate([np.asarray(s, np.uint64) for s in seed_sets])
                                 if len(seed_sets) else np.zeros(0, np.uint64))
    k = len(seed_sets)
    o, _ = _pr_opts(PageRank(pagerank.damping, pagerank.tol, pagerank.max_iter, pagerank.weighted))
    r = ranks_out if ranks_out is not None else np.zeros((k, graph.id_space), np.float64)
    it = iterations_out if iterations_out is not None else np.zeros(k, np.uint32)
    call, detail = _call()
    _raise(A.load().wc_ppr_batched(graph.handle, C.byref(call), C.byref(o), _ptr(nodes), _ptr(offs),
                                   k, _ptr(r), _ptr(it)), detail)
    return r, it


_KINDS = {"bfs": 0, "minplus": 1, "ppr": 2}


def set_schedule(graph: GraphVersion, kind: str, width: int, columns_per_pass: int,
                 blocks_per_sm: int = 4):
    s = A.Schedule(columns_per_pass, 1, blocks_per_sm, 0)
    _raise(A.load().wc_schedule_set(graph.handle, _KINDS[kind], width, C.byref(s)),
           A.ErrorDetail())


def autotune(graph: GraphVersion, kind: str, width: int) -> A.Schedule:
    s = A.Schedule()
    call, detail = _call()
    _raise(A.load().wc_autotune(graph.handle, C.byref(call), _KINDS[kind],
                                width, C.byref(s)), detail)
    return s


# ----------------------------------------------------------------- spectral


@dataclass
class EigenOptions:
    """spectral/lanczos.rs:136-168 with GraphMatrix (operator.rs:77-93)."""

    k: int
    which: str = "largest"
    operator: str = "adjacency"
    symmetrize: bool = True
    weighted: Optional[bool] = None
    tol: float = 1e-6
    max_iter: Optional[int] = None
    seed: int = 0


@dataclass
class Eigen:
    values: np.ndarray
    residuals: np.ndarray
    vectors: Optional[np.ndarray]
    iterations: int
    converged: bool
    components: int
    exact: int


_OPERATORS = ["adjacency", "laplacian", "normalized_laplacian", "random_walk"]


def eigen(graph: GraphVersion, options: EigenOptions, vectors=True) -> Eigen:
    """spectral/lanczos.rs:206-224 (f64 precision)."""
    o = A.EigenOpts(options.k, {"largest": 0, "smallest": 1}[options.which],
                    _OPERATORS.index(options.operator), int(options.symmetrize),
                    -1 if options.weighted is None else int(options.weighted), options.tol,
                    options.max_iter or 0, options.seed)
    k = options.k
    vals = np.zeros(k, np.float64)
    res = np.zeros(k, np.float64)
    vecs = np.zeros((k, graph.id_space), np.float64) if vectors else None
    st = A.EigenStats()
    call, detail = _call()
    _raise(A.load().wc_eigen(graph.handle, C.byref(call), C.byref(o), _ptr(vals), _ptr(res),
                             _ptr(vecs), C.byref(st)), detail)
    return Eigen(vals, res, vecs, st.iterations, bool(st.converged), st.components, st.exact)


# ----------------------------------------------------------------- adjoint


def pagerank_adjoint(graph: GraphVersion, loss_targets: Sequence[Sequence[int]],
                     pagerank: PageRank = PageRank(), adjoint_tol: float = 1e-14, grad_out=None):
    """∂L_c/∂w for L_c = Σ_{t in loss_targets[c]} x_t over every edge of the
    forward CSR: (grad[losses, edges], ranks, iterations)."""
    offs = np.zeros(len(loss_targets) + 1, np.uint64)
    for i, s in enumerate(loss_targets):
        offs[i + 1] = offs[i] + len(s)
    nodes = np.ascontiguousarray(np.concatenate([np.asarray(s, np.uint64) for s in loss_targets]))
    k = len(loss_targets)
    o, _ = _pr_opts(pagerank)
    g = grad_out if grad_out is not None else np.zeros((k, graph.edges), np.float64)
    ranks = np.zeros(graph.id_space, np.float64)
    it = np.zeros(2, np.uint32)
    call, detail = _call()
    _raise(A.load().wc_pagerank_adjoint(graph.handle, C.byref(call), C.byref(o), _ptr(nodes),
                                        _ptr(offs), k, adjoint_tol, _ptr(g), _ptr(ranks),
                                        _ptr(it)), detail)
    return g, ranks, it


# ----------------------------------------------------------------- ranking


def top_k(graph: GraphVersion, x, k: int, descending: bool = True, tombstones=None):
    """compute/ranking.rs:52: [(dense id, value)] best first."""
    nodes = np.zeros(max(k, 1), np.uint64)
    vals = np.zeros(max(k, 1), np.float64)
    count = C.c_uint64(0)
    call, detail = _call()
    _raise(A.load().wc_topk(graph.handle, C.byref(call), _dtype(x), _ptr(x), _ptr(tombstones), k,
                            int(descending), _ptr(nodes), _ptr(vals), C.byref(count)), detail)
    c = count.value
    return [(int(a), float(b)) for a, b in zip(nodes[:c], vals[:c])]


# ----------------------------------------------------------------- synthesis


@dataclass
class HostGraph:
    """A synthetic built version: CSR arrays and external ids by dense id."""

    offsets: np.ndarray
    targets: np.ndarray
    external_ids: np.ndarray
    weights: Optional[np.ndarray] = None

    @property
    def id_space(self) -> int:
        return len(self.offsets) - 1

    @property
    def edges(self) -> int:
        return len(self.targets)

    def upload(self, reverse=True, budget=None) -> GraphVersion:
        return GraphVersion(self.offsets, self.targets, self.weights, reverse, budget)


def _take(csr: A.HostCsr) -> HostGraph:
    n, m = csr.id_space, csr.edges
    off = np.ctypeslib.as_array(csr.offsets, shape=(n + 1,)).copy()
    tgt = np.ctypeslib.as_array(csr.targets, shape=(max(m, 1),))[:m].copy()
    ext = np.ctypeslib.as_array(csr.external_ids, shape=(max(n, 1),))[:n].copy()
    A.load().wc_host_csr_free(C.byref(csr))
    return HostGraph(off, tgt, ext)


def rmat(scale: int, edge_factor: int = 16, a: float = 0.57, b: float = 0.19, c: float = 0.19,
         seed: int = 1, undirected: bool = False) -> HostGraph:
    csr = A.HostCsr()
    _raise(A.load().wc_graph_rmat(scale, edge_factor, a, b, c, seed, int(undirected), C.byref(csr)),
           A.ErrorDetail())
    return _take(csr)


def gnm(n: int, m: int, seed: int = 1, undirected: bool = False) -> HostGraph:
    csr = A.HostCsr()
    _raise(A.load().wc_graph_gnm(n, m, seed, int(undirected), C.byref(csr)), A.ErrorDetail())
    return _take(csr)


def edge_weights(g: HostGraph, kind: str, seed: int = 7) -> np.ndarray:
    """Seeded per-edge weights as the benchmark configs define them:
    'uniform' U(0, 1]; 'int' integers U{1..100}; 'lognormal' exp(N(0, 1))
    row-normalised so each row sums to 1."""
    rng = np.random.default_rng(seed)
    m = g.edges
    if kind == "uniform":
        return 1.0 - rng.random(m)
    if kind == "int":
        return rng.integers(1, 101, m).astype(np.float64)
    if kind == "lognormal":
        w = np.exp(rng.standard_normal(m))
        deg = np.diff(g.offsets).astype(np.int64)
        rows = np.repeat(np.arange(g.id_space), deg)
        sums = np.bincount(rows, weights=w, minlength=g.id_space)
        return w / sums[rows]
    raise ValueError(kind)
