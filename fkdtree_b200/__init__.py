"""fkdtree_b200 -- the FKDTree flat kd-tree built and searched on B200 (sm_100a).

Python mirror of the reference's ``FKDTree<T, dim>`` interface (FKDTree.h:6-22,
FKDTree_cpu.h:16-327) over the C ABI of include/fkdtree_b200.h:

    tree = FKDTree(coords, ids)          # FKDTree_CPU(points) -- coords (dim, n) float32
    tree.build()                         # FKDTree_CPU::build
    tree.search_in_the_box(lo, hi)       # ids, in the reference's emission order
    tree.search_in_the_box_BFS(lo, hi)   # same list (the BFS variant emits the same order)
    tree.search_in_the_box_branchless(lo, hi)
    tree.search_in_the_box_recursive(lo, hi)   # same set; order: ascending heap index
    tree.search_in_the_box_multiple(mins, maxs)  # per-box counts (OpenCL backend semantics)
    tree.getDimensionVector(d), tree.getIdVector()

Batch entry points (``search_boxes``, ``count_boxes``, ``digest_boxes``) take
(dim, q) SoA boxes.  Inputs may be numpy arrays (host) or CUDA torch tensors
(device); everything runs on the GPU and there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import threading

import numpy as np

from . import _capi
from ._capi import FKDError, MEM_DEVICE, MEM_HOST, FLAG_ASYNC, check, lib

__all__ = ["FKDTree", "Batch", "MLP", "FKDError", "lib", "version"]


def version() -> str:
    return lib().fkd_version().decode()


def _is_torch(x) -> bool:
    return type(x).__module__.startswith("torch")


def _ptr(x):
    if x is None:
        return None
    if _is_torch(x):
        return C.c_void_p(x.data_ptr())
    return x.ctypes.data_as(C.c_void_p)


def _host_f32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float32)


_THREAD_BUFS = threading.local()


def _stream_handle(stream):
    if stream is None:
        return None
    if hasattr(stream, "cuda_stream"):
        return C.c_void_p(stream.cuda_stream)
    return C.c_void_p(int(stream))


class FKDTree:
    """The B200 tree.  ``coords`` is (dim, n) float32 SoA (numpy or CUDA
    tensor), ``ids`` (n,) uint32 (int32 tensors are reinterpreted); when ids are
    omitted they are 0..n-1, as in the reference drivers (main.cpp:182)."""

    def __init__(self, coords, ids=None, dim: int | None = None, stream=None, flags: int = 0):
        self._lib = lib()
        self.device = _is_torch(coords)
        if self.device:
            import torch
            coords = coords.contiguous()
            if coords.dtype != torch.float32:
                raise TypeError("coords must be float32")
            if ids is None:
                ids = torch.arange(coords.shape[1], dtype=torch.int32, device=coords.device)
            ids = ids.contiguous()
            if ids.dtype not in (torch.int32, torch.uint32):
                raise TypeError("ids must be a 32-bit integer tensor")
        else:
            coords = _host_f32(coords)
            if coords.ndim == 1:
                coords = coords.reshape(1, -1)
            ids = np.arange(coords.shape[1], dtype=np.uint32) if ids is None else np.ascontiguousarray(ids, dtype=np.uint32)
        self.dim = int(coords.shape[0]) if dim is None else int(dim)
        self.n = int(coords.shape[1])
        if ids.shape[0] != self.n:
            raise ValueError("ids and coords disagree on the number of points")
        self._coords, self._ids = coords, ids
        h = C.c_void_p()
        check(self._lib.fkd_create(self.dim, flags, _stream_handle(stream), C.byref(h)))
        self._h = h
        self._tables = None

    @classmethod
    def from_points(cls, points, dim: int, stream=None, flags: int = 0) -> "FKDTree":
        """A tree over points in the reference's FKDPoint<float, dim> layout
        (FKDPoint.h:102-103): n records of dim float32 coordinates then the
        uint32 id -- a numpy array or CUDA tensor of n * (dim + 1) 32-bit words
        (e.g. shape (n, dim + 1) float32 with the ids' bits in the last
        column).  build() passes them to fkd_build_points as they are."""
        self = cls.__new__(cls)
        self._lib = lib()
        self.device = _is_torch(points)
        if self.device:
            points = points.contiguous()
            words = points.numel() * points.element_size() // 4
        else:
            points = np.ascontiguousarray(points)
            words = points.nbytes // 4
        self.dim = int(dim)
        if words % (self.dim + 1):
            raise ValueError("points must hold n * (dim + 1) 32-bit words")
        self.n = words // (self.dim + 1)
        self._coords = self._ids = None
        self._points = points
        h = C.c_void_p()
        check(self._lib.fkd_create(self.dim, flags, _stream_handle(stream), C.byref(h)))
        self._h = h
        self._tables = None
        return self

    # -- FKDTree_CPU::build (FKDTree_cpu.h:221-277)
    def build(self) -> "FKDTree":
        mem = MEM_DEVICE if self.device else MEM_HOST
        if getattr(self, "_points", None) is not None:
            check(self._lib.fkd_build_points(self._h, _ptr(self._points), self.n, mem))
        else:
            check(self._lib.fkd_build(self._h, _ptr(self._coords), _ptr(self._ids), self.n, mem))
        self._tables = None
        return self

    # -- getDimensionVector / getIdVector (FKDTree_cpu.h:209-213)
    def tables(self) -> tuple[np.ndarray, np.ndarray]:
        if self._tables is None:
            tab = np.empty((self.dim, self.n), dtype=np.float32)
            tid = np.empty(self.n, dtype=np.uint32)
            check(self._lib.fkd_get_tables(self._h, _ptr(tab), _ptr(tid), MEM_HOST))
            self._tables = (tab, tid)
        return self._tables

    def getDimensionVector(self, dimension: int) -> np.ndarray:
        tab, _ = self.tables()
        return tab[dimension] if 0 <= dimension < self.dim else tab[0]  # FKDTree_cpu.h:210-211

    def getIdVector(self) -> np.ndarray:
        return self.tables()[1]

    # -- batched searches over (dim, q) SoA boxes
    def _boxes(self, mins, maxs):
        if _is_torch(mins):
            return mins.contiguous(), maxs.contiguous(), MEM_DEVICE, int(mins.shape[-1])
        mins = _host_f32(mins).reshape(self.dim, -1)
        maxs = _host_f32(maxs).reshape(self.dim, -1)
        return mins, maxs, MEM_HOST, int(mins.shape[1])

    def count_boxes(self, mins, maxs) -> np.ndarray:
        mins, maxs, mem, q = self._boxes(mins, maxs)
        if mem == MEM_DEVICE:
            import torch
            counts = torch.empty(q, dtype=torch.int32, device=mins.device)
        else:
            counts = np.empty(q, dtype=np.uint32)
        check(self._lib.fkd_search_count(self._h, _ptr(mins), _ptr(maxs), q, _ptr(counts), mem))
        return counts

    def search_boxes(self, mins, maxs, ordered: bool = True, capacity: int | None = None):
        """Returns (offsets (q+1,) uint64, ids) with the ids of box j in
        ids[offsets[j]:offsets[j+1]]; ``ordered`` gives the reference's
        emission order (ascending heap index)."""
        mins, maxs, mem, q = self._boxes(mins, maxs)
        total = C.c_uint64(0)
        if mem == MEM_DEVICE:
            import torch
            counts = self.count_boxes(mins, maxs)
            offsets = torch.zeros(q + 1, dtype=torch.int64, device=mins.device)
            offsets[1:] = torch.cumsum(counts.to(torch.int64), 0)
            tot = int(offsets[-1].item())
            out = torch.empty(max(tot, 1), dtype=torch.int32, device=mins.device)
            check(self._lib.fkd_search_write(self._h, _ptr(mins), _ptr(maxs), q, _ptr(offsets), _ptr(out),
                                             int(ordered), mem))
            return offsets, out[:tot]
        offsets = np.empty(q + 1, dtype=np.uint64)
        if capacity is None:
            counts = self.count_boxes(mins, maxs)
            capacity = int(counts.sum(dtype=np.uint64))
        out = np.empty(max(capacity, 1), dtype=np.uint32)
        check(self._lib.fkd_search(self._h, _ptr(mins), _ptr(maxs), q, _ptr(offsets), _ptr(out), capacity,
                                   C.byref(total), int(ordered), mem))
        return offsets, out[:total.value]

    def digest_boxes(self, mins, maxs):
        mins, maxs, mem, q = self._boxes(mins, maxs)
        if mem == MEM_DEVICE:
            import torch
            counts = torch.empty(q, dtype=torch.int32, device=mins.device)
            dig = torch.empty(q, dtype=torch.int64, device=mins.device)
        else:
            counts = np.empty(q, dtype=np.uint32)
            dig = np.empty(q, dtype=np.uint64)
        check(self._lib.fkd_search_digest(self._h, _ptr(mins), _ptr(maxs), q, _ptr(counts), _ptr(dig), mem))
        return counts, dig

    # -- single-box searches, the reference's per-query API
    def _one(self, minPoint, maxPoint, ordered=True) -> np.ndarray:
        """One box in one library call: the ids land in a per-thread buffer
        sized by the largest box seen so far (a larger box takes a second call
        with the total fkd_search reports).  Safe from several threads at once."""
        lo = _host_f32(minPoint).reshape(self.dim, 1)
        hi = _host_f32(maxPoint).reshape(self.dim, 1)
        tl = _THREAD_BUFS.__dict__
        buf = tl.get("buf")
        if buf is None:
            buf = tl["buf"] = np.empty(256, dtype=np.uint32)
        offs = np.zeros(2, dtype=np.uint64)
        total = C.c_uint64(0)
        args = (self._h, _ptr(lo), _ptr(hi), 1, _ptr(offs))
        st = self._lib.fkd_search(*args, _ptr(buf), buf.size, C.byref(total), int(ordered), MEM_HOST)
        if st == _capi.ERR_CAPACITY and total.value > buf.size:
            buf = tl["buf"] = np.empty(total.value + total.value // 2, dtype=np.uint32)
            st = self._lib.fkd_search(*args, _ptr(buf), buf.size, C.byref(total), int(ordered), MEM_HOST)
        check(st)
        return buf[:total.value].copy()

    def search_in_the_box(self, minPoint, maxPoint) -> np.ndarray:  # FKDTree_cpu.h:123-169
        return self._one(minPoint, maxPoint)

    def search_in_the_box_BFS(self, minPoint, maxPoint) -> np.ndarray:  # FKDTree_cpu.h:72-121
        return self._one(minPoint, maxPoint)

    def search_in_the_box_branchless(self, minPoint, maxPoint) -> np.ndarray:  # FKDTree_cpu.h:25-70
        return self._one(minPoint, maxPoint)

    def search_in_the_box_recursive(self, minPoint, maxPoint) -> np.ndarray:  # FKDTree_cpu.h:171-207
        return self._one(minPoint, maxPoint)

    def search_in_the_box_multiple(self, minPoints, maxPoints) -> np.ndarray:
        """Per-box result counts, the OpenCL backend's semantics
        (FKDTree_opencl.h:123-164); the CPU backend's stub returns nothing
        (FKDTree_cpu.h:215-219)."""
        return self.count_boxes(minPoints, maxPoints)

    # -- radius and k-nearest-neighbour search (fkd_nn.cu; no reference counterpart)
    def _centres(self, centres):
        if _is_torch(centres):
            return centres.contiguous(), MEM_DEVICE, int(centres.shape[-1])
        centres = _host_f32(centres).reshape(self.dim, -1)
        return centres, MEM_HOST, int(centres.shape[1])

    def _radii(self, radii, q, mem, like):
        if mem == MEM_DEVICE:
            import torch
            r = radii if _is_torch(radii) else torch.as_tensor(np.asarray(radii, dtype=np.float32))
            r = r.to(device=like.device, dtype=torch.float32)
            return r.expand(q).contiguous() if r.dim() == 0 or r.numel() == 1 else r.contiguous()
        r = _host_f32(radii).reshape(-1)
        return np.full(q, r[0], dtype=np.float32) if r.size == 1 else r

    def count_radius(self, centres, radii):
        """Points within radii[j] (inclusive) of every centre (dim, q); radii
        is (q,) or one value."""
        ctr, mem, q = self._centres(centres)
        rad = self._radii(radii, q, mem, ctr)
        if mem == MEM_DEVICE:
            import torch
            counts = torch.empty(q, dtype=torch.int32, device=ctr.device)
        else:
            counts = np.empty(q, dtype=np.uint32)
        check(self._lib.fkd_search_radius_count(self._h, _ptr(ctr), _ptr(rad), q, _ptr(counts), mem))
        return counts

    def search_radius(self, centres, radii, ordered: bool = True, capacity: int | None = None):
        """Returns (offsets (q+1,), ids): the ids of query j are
        ids[offsets[j]:offsets[j+1]], in ascending heap index when ``ordered``
        (else in the walk's depth-first order)."""
        ctr, mem, q = self._centres(centres)
        rad = self._radii(radii, q, mem, ctr)
        if capacity is None:
            counts = self.count_radius(ctr, rad)
            capacity = int(counts.sum().item()) if mem == MEM_DEVICE else int(counts.sum(dtype=np.uint64))
        total = C.c_uint64(0)
        if mem == MEM_DEVICE:
            import torch
            offsets = torch.empty(q + 1, dtype=torch.int64, device=ctr.device)
            out = torch.empty(max(capacity, 1), dtype=torch.int32, device=ctr.device)
        else:
            offsets = np.empty(q + 1, dtype=np.uint64)
            out = np.empty(max(capacity, 1), dtype=np.uint32)
        check(self._lib.fkd_search_radius(self._h, _ptr(ctr), _ptr(rad), q, _ptr(offsets), _ptr(out), capacity,
                                          C.byref(total), int(ordered), mem))
        return offsets, out[:total.value]

    def knn(self, centres, k: int):
        """The k nearest points of every centre (dim, q), ascending in
        (squared distance, id): returns (ids (q, k), d2 (q, k)); missing
        neighbours are id 0xffffffff with d2 = inf."""
        ctr, mem, q = self._centres(centres)
        if mem == MEM_DEVICE:
            import torch
            ids = torch.empty((q, k), dtype=torch.int32, device=ctr.device)
            d2 = torch.empty((q, k), dtype=torch.float32, device=ctr.device)
        else:
            ids = np.empty((q, k), dtype=np.uint32)
            d2 = np.empty((q, k), dtype=np.float32)
        check(self._lib.fkd_search_knn(self._h, _ptr(ctr), q, int(k), _ptr(ids), _ptr(d2), mem))
        return ids, d2

    def set_param(self, name: str, value: int) -> "FKDTree":
        """Tuning knob ("hist_ctas", "search_lanes"; fkd_set_param)."""
        check(self._lib.fkd_set_param(self._h, name.encode(), int(value)))
        return self

    def set_mlp(self, mlp, delta: float = 0.05) -> "FKDTree":
        """Learned split for later builds (None: plain radix select)."""
        self._mlp = mlp
        check(self._lib.fkd_set_mlp(self._h, mlp._h if mlp else None, float(delta)))
        return self

    def learn_stats(self, reset: bool = False) -> dict:
        st = np.zeros(4, dtype=np.uint64)
        check(self._lib.fkd_learn_stats(self._h, _ptr(st), int(reset)))
        return dict(brackets=int(st[0]), verified=int(st[1]), fallbacks=int(st[2]), passes=int(st[3]))

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.fkd_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Many independent events built and searched together (fkd_batch_* in
    include/fkdtree_b200.h).  ``dims`` (E,), ``pt_off`` / ``q_off`` (E+1,)
    describe the layout of fkdtree_b200.workloads.Batch: event e owns points
    [pt_off[e], pt_off[e+1]) and boxes [q_off[e], q_off[e+1]); its coordinates
    (and boxes) are an SoA slice of the flat arrays."""

    def __init__(self, dims, pt_off, q_off, stream=None, flags: int = 0):
        self._lib = lib()
        self.dims = np.ascontiguousarray(dims, dtype=np.uint32)
        self.pt_off = np.ascontiguousarray(pt_off, dtype=np.uint64)
        self.q_off = np.ascontiguousarray(q_off, dtype=np.uint64)
        self.n_events = int(self.dims.shape[0])
        n = np.diff(self.pt_off.astype(np.int64))
        self.n_coords = int((n * self.dims).sum())
        self.n_points = int(self.pt_off[-1])
        self.n_boxes = int(self.q_off[-1])
        h = C.c_void_p()
        check(self._lib.fkd_batch_create(self.n_events, _ptr(self.dims), _ptr(self.pt_off), _ptr(self.q_off), flags,
                                         _stream_handle(stream), C.byref(h)))
        self._h = h

    @classmethod
    def of(cls, wb, **kw) -> "Batch":
        return cls(wb.dims, wb.pt_off, wb.q_off, **kw)

    def set_param(self, name: str, value: int) -> None:
        check(self._lib.fkd_batch_set_param(self._h, name.encode(), int(value)))

    def autotune(self, coords, ids, mins, maxs, **kw) -> dict:
        """Sweeps the launch knobs on these inputs and keeps the fastest
        (fkdtree_b200.autotune.tune_batch)."""
        from . import autotune
        return autotune.tune_batch(self, coords, ids, mins, maxs, **kw)

    def build(self, coords, ids) -> "Batch":
        if _is_torch(coords):
            check(self._lib.fkd_batch_build(self._h, _ptr(coords), _ptr(ids), MEM_DEVICE))
        else:
            c = _host_f32(coords)
            i = np.ascontiguousarray(ids, dtype=np.uint32)
            check(self._lib.fkd_batch_build(self._h, _ptr(c), _ptr(i), MEM_HOST))
        return self

    def tables(self):
        tab = np.empty(self.n_coords, dtype=np.float32)
        tid = np.empty(self.n_points, dtype=np.uint32)
        check(self._lib.fkd_batch_get_tables(self._h, _ptr(tab), _ptr(tid), MEM_HOST))
        return tab, tid

    def search_digest(self, mins, maxs):
        if _is_torch(mins):
            import torch
            counts = torch.empty(self.n_boxes, dtype=torch.int32, device=mins.device)
            dig = torch.empty(self.n_boxes, dtype=torch.int64, device=mins.device)
            check(self._lib.fkd_batch_search_digest(self._h, _ptr(mins), _ptr(maxs), _ptr(counts), _ptr(dig),
                                                    MEM_DEVICE))
            return counts, dig
        lo, hi = _host_f32(mins), _host_f32(maxs)
        counts = np.empty(self.n_boxes, dtype=np.uint32)
        dig = np.empty(self.n_boxes, dtype=np.uint64)
        check(self._lib.fkd_batch_search_digest(self._h, _ptr(lo), _ptr(hi), _ptr(counts), _ptr(dig), MEM_HOST))
        return counts, dig

    def set_mlp(self, mlp, delta: float = 0.05) -> "Batch":
        self._mlp = mlp
        check(self._lib.fkd_batch_set_mlp(self._h, mlp._h if mlp else None, float(delta)))
        return self

    def learn_stats(self, reset: bool = False) -> dict:
        st = np.zeros(4, dtype=np.uint64)
        check(self._lib.fkd_batch_learn_stats(self._h, _ptr(st), int(reset)))
        return dict(brackets=int(st[0]), verified=int(st[1]), fallbacks=int(st[2]), passes=int(st[3]))

    def record(self, coords, ids, cap: int | None = None):
        """Exact build that records (features, target) of every globally split
        node; returns (x (m, 40) float32, t (m,) float32)."""
        cap = cap if cap is not None else max(1024, self.n_points // 512)
        x = np.empty((cap, MLP.IN), dtype=np.float32)
        t = np.empty(cap, dtype=np.float32)
        n = C.c_uint64(0)
        if _is_torch(coords):
            check(self._lib.fkd_batch_record(self._h, _ptr(coords), _ptr(ids), _ptr(x), _ptr(t), cap, C.byref(n),
                                             MEM_DEVICE))
        else:
            c = _host_f32(coords)
            i = np.ascontiguousarray(ids, dtype=np.uint32)
            check(self._lib.fkd_batch_record(self._h, _ptr(c), _ptr(i), _ptr(x), _ptr(t), cap, C.byref(n), MEM_HOST))
        m = min(int(n.value), cap)
        return x[:m], t[:m]

    def run(self, coords, ids, mins, maxs, counts, digests) -> None:
        """Build + digest search of CUDA tensors as one CUDA graph launch."""
        check(self._lib.fkd_batch_run(self._h, _ptr(coords), _ptr(ids), _ptr(mins), _ptr(maxs), _ptr(counts),
                                      _ptr(digests)))

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.fkd_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class MLP:
    """The learned split predictor (fkd_mlp_* in include/fkdtree_b200.h):
    40 -> 64 -> 64 -> 1, GELU, bf16 tensor-core products with fp32
    accumulation, trained on the GPU."""

    IN = 40

    def __init__(self, seed: int = 0):
        self._lib = lib()
        h = C.c_void_p()
        check(self._lib.fkd_mlp_create(seed, C.byref(h)))
        self._h = h
        self.n_params = int(self._lib.fkd_mlp_param_count())

    @property
    def params(self) -> np.ndarray:
        p = np.empty(self.n_params, dtype=np.float32)
        check(self._lib.fkd_mlp_get_params(self._h, _ptr(p)))
        return p

    @params.setter
    def params(self, p) -> None:
        p = np.ascontiguousarray(p, dtype=np.float32)
        assert p.shape == (self.n_params,)
        check(self._lib.fkd_mlp_set_params(self._h, _ptr(p)))

    def forward(self, x) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float32).reshape(-1, self.IN)
        y = np.empty(x.shape[0], dtype=np.float32)
        check(self._lib.fkd_mlp_forward(self._h, _ptr(x), x.shape[0], _ptr(y), MEM_HOST))
        return y

    def grad(self, x, t):
        x = np.ascontiguousarray(x, dtype=np.float32).reshape(-1, self.IN)
        t = np.ascontiguousarray(t, dtype=np.float32)
        g = np.empty(self.n_params, dtype=np.float32)
        loss = C.c_float(0.0)
        check(self._lib.fkd_mlp_grad(self._h, _ptr(x), _ptr(t), x.shape[0], _ptr(g), C.byref(loss), MEM_HOST))
        return g, float(loss.value)

    def save(self, path, storage: str = "f32") -> None:
        """Writes the parameters to a versioned weights file
        (fkdtree_b200.mlp_file; "f32" exact, "bf16" half the size)."""
        from . import mlp_file
        mlp_file.save_params(path, self.params, storage)

    @classmethod
    def load(cls, path) -> "MLP":
        """A network with the parameters of a weights file written by save()."""
        from . import mlp_file
        m = cls()
        m.params = mlp_file.load_params(path)
        return m

    def train(self, x, t, epochs: int = 30, batch: int = 256, lr: float = 2e-3, seed: int = 0) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float32).reshape(-1, self.IN)
        t = np.ascontiguousarray(t, dtype=np.float32)
        losses = np.empty(epochs, dtype=np.float32)
        check(self._lib.fkd_mlp_train(self._h, _ptr(x), _ptr(t), x.shape[0], epochs, batch, float(lr), seed,
                                      _ptr(losses), MEM_HOST))
        return losses

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.fkd_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
