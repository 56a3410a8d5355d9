"""Host-side mirror of the reference's solver interface over the C ABI.

Three classes keep the reference's names, argument meanings and strings, so a
caller of the reference switches by changing an import:

* ``TdmaBackendGPU``  — the runtime backend selector of the heat app
  (apps/heat_gpu/tdma_backend_gpu.hpp:21-70): ``parse("pascal" | "pascal_tdma" |
  "filtered_v2" | anything else -> FILTERED)``, ``solve``, ``solve_cyclic``,
  ``set_rho_device``, ``set_eps_constant``, ``last_comm_ms``, ``last_gpu_ms``.
* ``PaScaLTDMACUDA``  — libs/pascal_tdma/include/pascal_tdma_cuda.hpp:18-56.
* ``FilteredTDMACUDA`` — libs/filtered_tdma/include/filtered_tdma_cuda.hpp:161-266.

Arrays are torch CUDA tensors (float64, [n_row, n_sys] C-contiguous) or raw
device pointers; torch is only the allocator and stream provider.  The MPI
arguments of the reference constructors are accepted and ignored except
``nprocs``, which becomes the number of segments P each system is split into
inside the GPU.  ``last_comm_ms()`` is always 0: there is no communication.

``Solver`` is the plain handle wrapper the three classes are built on.
"""
from __future__ import annotations

import ctypes
from enum import Enum

from . import _lib as L

try:
    import torch
except ImportError:  # raw-pointer use without torch
    torch = None

MPI_PROC_NULL = -2


def _ptr(x) -> int:
    if isinstance(x, int):
        return x
    if torch is not None and isinstance(x, torch.Tensor):
        if not x.is_cuda:
            raise ValueError("arrays must be CUDA tensors (device pointers)")
        if not x.is_contiguous():
            raise ValueError("arrays must be contiguous [n_row, n_sys]")
        return x.data_ptr()
    raise TypeError(f"expected a CUDA tensor or a device pointer, got {type(x)}")


def _shape(x, n_sys, n_row):
    if n_sys is not None and n_row is not None:
        return int(n_sys), int(n_row)
    if torch is not None and isinstance(x, torch.Tensor) and x.dim() == 2:
        return int(x.shape[1]), int(x.shape[0])
    raise ValueError("n_sys and n_row are required with raw pointers")


def _stream(stream) -> int:
    if stream is None:
        if torch is not None and torch.cuda.is_available():
            return torch.cuda.current_stream().cuda_stream
        return 0
    if isinstance(stream, int):
        return stream
    return stream.cuda_stream


def _check_dtype(*xs, dtype=None):
    if torch is None:
        return
    want = dtype or torch.float64
    for x in xs:
        if isinstance(x, torch.Tensor) and x.dtype != want:
            raise TypeError(f"expected {want} arrays, got {x.dtype}")


def _ragged_host(row_offsets, periodic):
    import numpy as np
    off = np.ascontiguousarray(row_offsets, dtype=np.int64)
    n_sys = off.shape[0] - 1
    per = None
    if periodic is not None:
        per = np.ascontiguousarray(periodic, dtype=np.uint8)
        if per.shape[0] != n_sys:
            raise ValueError("periodic needs one flag per system")
    return off, per, n_sys


class Solver:
    """One btdma handle: method, capacity (n_sys, n_row), segments P."""

    METHODS = {"pascal": L.PASCAL, "filtered_v1": L.FILTERED_V1, "filtered_v2": L.FILTERED_V2}

    def __init__(self, method="pascal", n_sys=1, n_row=3, P=0, precision=L.FP64, flags=0):
        m = self.METHODS[method] if isinstance(method, str) else int(method)
        h = ctypes.c_void_p()
        L.check(L.lib().btdma_create(m, int(n_sys), int(n_row), int(P), int(precision),
                                     int(flags), ctypes.byref(h)))
        self._h = h
        self.method = m
        self.n_sys, self.n_row = int(n_sys), int(n_row)
        p = ctypes.c_int()
        L.check(L.lib().btdma_segments(h, ctypes.byref(p)))
        self.P = p.value

    def close(self):
        if getattr(self, "_h", None):
            L.lib().btdma_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_method(self, method):
        m = self.METHODS[method] if isinstance(method, str) else int(method)
        L.check(L.lib().btdma_set_method(self._h, m))
        self.method = m

    def solve(self, A, B, C, D, n_sys=None, n_row=None, stream=None, cyclic=False):
        """In place: D <- x."""
        _check_dtype(A, B, C, D)
        ns, nr = _shape(D, n_sys, n_row)
        f = L.lib().btdma_solve_cyclic if cyclic else L.lib().btdma_solve
        L.check(f(self._h, _ptr(A), _ptr(B), _ptr(C), _ptr(D), ns, nr, _stream(stream)))
        return D

    def solve_out(self, A, B, C, D, X, n_sys=None, n_row=None, stream=None, cyclic=False):
        """X <- x; D unchanged."""
        _check_dtype(A, B, C, D, X)
        ns, nr = _shape(D, n_sys, n_row)
        L.check(L.lib().btdma_solve_out(self._h, _ptr(A), _ptr(B), _ptr(C), _ptr(D), _ptr(X),
                                        ns, nr, int(cyclic), _stream(stream)))
        return X

    def solve_host(self, A, B, C, D, X, n_sys=None, n_row=None, stream=None, cyclic=False):
        """X <- x for a batch in host memory (CPU float64 tensors [n_row, n_sys],
        pinned for overlapping copies; btdma_solve_host).  D unchanged."""
        if torch is None:
            raise RuntimeError("solve_host takes torch CPU tensors")
        _check_dtype(A, B, C, D, X)
        for x in (A, B, C, D, X):
            if not isinstance(x, torch.Tensor) or x.is_cuda or not x.is_contiguous():
                raise ValueError("solve_host takes contiguous CPU tensors [n_row, n_sys]")
        ns, nr = _shape(D, n_sys, n_row)
        for x in (A, B, C, D, X):
            if x.numel() < ns * nr:
                raise ValueError("host array smaller than n_row * n_sys")
        L.check(L.lib().btdma_solve_host(self._h, A.data_ptr(), B.data_ptr(), C.data_ptr(),
                                         D.data_ptr(), X.data_ptr(), ns, nr, int(cyclic),
                                         _stream(stream)))
        return X

    def solve_f32(self, A, B, C, D, X, n_sys=None, n_row=None, stream=None, cyclic=False):
        """FP32-stored A, B, C, D (handle precision FP32_STORE or FP32_REFINE); X <- x in FP64."""
        if torch is not None:
            _check_dtype(A, B, C, D, dtype=torch.float32)
            _check_dtype(X)
        ns, nr = _shape(D, n_sys, n_row)
        L.check(L.lib().btdma_solve_f32(self._h, _ptr(A), _ptr(B), _ptr(C), _ptr(D), _ptr(X),
                                        ns, nr, int(cyclic), _stream(stream)))
        return X

    def solve_ragged(self, A, B, C, D, X, row_offsets, periodic=None, stream=None):
        """Ragged batch (CSR layout, see btdma_solve_ragged): A..D are 1-D device
        arrays (float64, or float32 with an FP32 handle), X float64; row_offsets
        (n_sys + 1, int64) and periodic (n_sys, uint8 or None) are host arrays."""
        off, per, n_sys = _ragged_host(row_offsets, periodic)
        f32 = torch is not None and isinstance(A, torch.Tensor) and A.dtype == torch.float32
        if torch is not None:
            _check_dtype(A, B, C, D, dtype=torch.float32 if f32 else torch.float64)
            _check_dtype(X)
        f = L.lib().btdma_solve_ragged_f32 if f32 else L.lib().btdma_solve_ragged
        L.check(f(self._h, _ptr(A), _ptr(B), _ptr(C), _ptr(D), _ptr(X), off.ctypes.data,
                  per.ctypes.data if per is not None else None, n_sys, _stream(stream)))
        return X

    def ragged_autotune(self, A, B, C, D, X, row_offsets, periodic=None, stream=None):
        """Pick lanes per system and warps per CTA for every length bucket by
        timing them on this batch (X is overwritten); returns the plan."""
        off, per, n_sys = _ragged_host(row_offsets, periodic)
        L.check(L.lib().btdma_ragged_autotune(
            self._h, _ptr(A), _ptr(B), _ptr(C), _ptr(D), _ptr(X), off.ctypes.data,
            per.ctypes.data if per is not None else None, n_sys, _stream(stream)))
        return self.ragged_plan()

    def ragged_plan(self) -> list:
        n = ctypes.c_int()
        L.check(L.lib().btdma_ragged_plan_info(self._h, None, 0, ctypes.byref(n)))
        arr = (L.RaggedBucket * max(1, n.value))()
        L.check(L.lib().btdma_ragged_plan_info(self._h, arr, n.value, ctypes.byref(n)))
        return [arr[i].as_dict() for i in range(n.value)]

    def ragged_set_plan(self, plan):
        """Apply launch shapes (a list of ragged_plan() dicts, in its order) to the
        current ragged plan; see btdma_ragged_set_plan."""
        arr = (L.RaggedBucket * max(1, len(plan)))()
        for i, b in enumerate(plan):
            for f, _ in L.RaggedBucket._fields_:
                setattr(arr[i], f, b[f])
        L.check(L.lib().btdma_ragged_set_plan(self._h, arr, len(plan)))

    def set_tile_shape(self, shape):
        """Kernel shape of the tiled PaScaL solves: TILE_AUTO, TILE_NARROW or
        TILE_WIDE (same results; see btdma_set_tile_shape)."""
        L.check(L.lib().btdma_set_tile_shape(self._h, int(shape)))

    def set_refine(self, max_sweeps=3, eta_tol=8 * 2.0**-53):
        """Refinement sweeps and backward-error bound of an FP32_REFINE handle."""
        L.check(L.lib().btdma_set_refine(self._h, int(max_sweeps), float(eta_tol)))

    def last_stats(self) -> dict:
        """Refinement statistics of the most recent solve (blocking read)."""
        st = L.Stats()
        L.check(L.lib().btdma_last_stats(self._h, ctypes.byref(st)))
        return st.as_dict()

    def set_eps_constant(self, eps_constant):
        L.check(L.lib().btdma_set_eps_constant(self._h, float(eps_constant)))

    def set_rho(self, A, B, C, n_sys=None, n_row=None, stream=None, all_systems=False):
        ns, nr = _shape(A, n_sys, n_row)
        f = L.lib().btdma_set_rho_all if all_systems else L.lib().btdma_set_rho
        L.check(f(self._h, _ptr(A), _ptr(B), _ptr(C), ns, nr, _stream(stream)))

    def last_J(self):
        buf = (ctypes.c_int * max(1, self.P))()
        n = ctypes.c_int()
        L.check(L.lib().btdma_last_J(self._h, buf, self.P, ctypes.byref(n)))
        return list(buf)[: n.value]

    def status(self) -> int:
        st = ctypes.c_uint()
        L.check(L.lib().btdma_status(self._h, ctypes.byref(st)))
        return st.value


class _Timed:
    """CUDA-event timing of the last profiled solve (last_gpu_ms)."""

    def __init__(self):
        self._gpu_ms = 0.0

    def _timed(self, fn):
        if torch is None:
            fn()
            return
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        fn()
        e1.record()
        e1.synchronize()
        self._gpu_ms = float(e0.elapsed_time(e1))

    def last_comm_ms(self) -> float:
        return 0.0

    def last_gpu_ms(self) -> float:
        return self._gpu_ms


class PaScaLTDMACUDA(_Timed):
    """Exact P-segment solver (libs/pascal_tdma/include/pascal_tdma_cuda.hpp:18-56).

    ``nprocs`` is the segment count P; ``myrank``, ``comm``, ``block_x``,
    ``block_y`` are accepted for signature compatibility.  The device handle is
    created on the first solve, when n_row is known, and re-created only if a
    later solve needs more rows.
    """

    def __init__(self, n_sys, myrank=0, nprocs=1, comm=None, block_x=128, block_y=1):
        super().__init__()
        self._n_sys, self._nprocs = int(n_sys), int(nprocs)
        self._solver = None

    def _get(self, n_sys, n_row):
        s = self._solver
        if s is None or n_row > s.n_row or n_sys > s.n_sys:
            if s is not None:
                s.close()
            s = self._solver = Solver("pascal", max(n_sys, self._n_sys), n_row, self._nprocs)
        return s

    def solve(self, d_A, d_B, d_C, d_D, n_sys, n_row):
        self._get(n_sys, n_row).solve(d_A, d_B, d_C, d_D, n_sys, n_row)

    def solve_cyclic(self, d_A, d_B, d_C, d_D, n_sys, n_row):
        self._get(n_sys, n_row).solve(d_A, d_B, d_C, d_D, n_sys, n_row, cyclic=True)

    def solve_profile(self, d_A, d_B, d_C, d_D, n_sys, n_row):
        self._timed(lambda: self.solve(d_A, d_B, d_C, d_D, n_sys, n_row))

    def solve_cyclic_profile(self, d_A, d_B, d_C, d_D, n_sys, n_row):
        self._timed(lambda: self.solve_cyclic(d_A, d_B, d_C, d_D, n_sys, n_row))

    def nprocs(self):
        return self._nprocs

    def n_sys_rt(self):
        return self._n_sys

    def n_row_rt(self):
        return 2 * self._nprocs


class FilteredTDMACUDA(_Timed):
    """Filtered P-segment solver (libs/filtered_tdma/include/filtered_tdma_cuda.hpp:161-266)."""

    def __init__(self, n_sys, n_row, myrank=0, nprocs=1, comm=None,
                 left_rank=MPI_PROC_NULL, right_rank=MPI_PROC_NULL, eps_constant=1.0e-12,
                 flags=0):
        super().__init__()
        self._n_sys, self._n_row, self._nprocs = int(n_sys), int(n_row), int(nprocs)
        self._solver = Solver("filtered_v2", n_sys, n_row, nprocs, flags=flags)
        self._solver.set_eps_constant(eps_constant)

    def _run(self, method, A, B, C, D, cyclic):
        self._solver.set_method(method)
        self._solver.solve(A, B, C, D, self._n_sys, self._n_row, cyclic=cyclic)

    def solve_filtered_v1(self, d_A, d_B, d_C, d_D):
        self._run(L.FILTERED_V1, d_A, d_B, d_C, d_D, False)

    def solve_filtered_v2(self, d_A, d_B, d_C, d_D):
        self._run(L.FILTERED_V2, d_A, d_B, d_C, d_D, False)

    def solve_cycl_filtered_v1(self, d_A, d_B, d_C, d_D):
        self._run(L.FILTERED_V1, d_A, d_B, d_C, d_D, True)

    def solve_cycl_filtered_v2(self, d_A, d_B, d_C, d_D):
        self._run(L.FILTERED_V2, d_A, d_B, d_C, d_D, True)

    def solve_filtered_v1_profile(self, *a):
        self._timed(lambda: self.solve_filtered_v1(*a))

    def solve_filtered_v2_profile(self, *a):
        self._timed(lambda: self.solve_filtered_v2(*a))

    def solve_cycl_filtered_v1_profile(self, *a):
        self._timed(lambda: self.solve_cycl_filtered_v1(*a))

    def solve_cycl_filtered_v2_profile(self, *a):
        self._timed(lambda: self.solve_cycl_filtered_v2(*a))

    def set_rho_device(self, d_A, d_B, d_C):
        self._solver.set_rho(d_A, d_B, d_C, self._n_sys, self._n_row)

    def set_eps_constant(self, eps_constant):
        self._solver.set_eps_constant(eps_constant)

    def last_J(self) -> int:
        """J of the first segment (the reference reports its rank's own J)."""
        return self._solver.last_J()[0]

    def last_J_all(self):
        return self._solver.last_J()

    def n_sys(self):
        return self._n_sys

    def n_row(self):
        return self._n_row

    def nprocs(self):
        return self._nprocs


class TdmaBackendGPU(_Timed):
    """Runtime backend selector (apps/heat_gpu/tdma_backend_gpu.hpp:21-70)."""

    class Kind(Enum):
        FILTERED = 0
        FILTERED_V2 = 1
        PASCAL = 2

    @staticmethod
    def parse(s: str) -> "TdmaBackendGPU.Kind":
        """Case-insensitive, as apps/heat_gpu/tdma_backend_gpu.cu:6-13."""
        t = s.lower()
        if t in ("pascal", "pascal_tdma"):
            return TdmaBackendGPU.Kind.PASCAL
        if t == "filtered_v2":
            return TdmaBackendGPU.Kind.FILTERED_V2
        return TdmaBackendGPU.Kind.FILTERED

    def __init__(self, kind, n_sys, n_row, myrank=0, nprocs=1, comm=None,
                 left_rank=MPI_PROC_NULL, right_rank=MPI_PROC_NULL, eps_constant=1.0e-12):
        super().__init__()
        if isinstance(kind, str):
            kind = self.parse(kind)
        self._kind = kind
        self._n_sys, self._n_row = int(n_sys), int(n_row)
        if kind == self.Kind.PASCAL:
            self._pasc = PaScaLTDMACUDA(n_sys, myrank, nprocs, comm)
            self._filt = None
        else:
            self._filt = FilteredTDMACUDA(n_sys, n_row, myrank, nprocs, comm, left_rank,
                                          right_rank, eps_constant)
            self._pasc = None

    def kind(self):
        return self._kind

    def solve(self, d_A, d_B, d_C, d_D):
        """The heat app's benchmark path: every backend through its profile variant
        (tdma_backend_gpu.cu:35-46), so last_gpu_ms() is populated."""
        if self._kind == self.Kind.FILTERED:
            self._filt.solve_filtered_v1_profile(d_A, d_B, d_C, d_D)
        elif self._kind == self.Kind.FILTERED_V2:
            self._filt.solve_filtered_v2_profile(d_A, d_B, d_C, d_D)
        else:
            self._pasc.solve_profile(d_A, d_B, d_C, d_D, self._n_sys, self._n_row)

    def solve_cyclic(self, d_A, d_B, d_C, d_D):
        if self._kind == self.Kind.FILTERED:
            self._filt.solve_cycl_filtered_v1_profile(d_A, d_B, d_C, d_D)
        elif self._kind == self.Kind.FILTERED_V2:
            self._filt.solve_cycl_filtered_v2_profile(d_A, d_B, d_C, d_D)
        else:
            self._pasc.solve_cyclic_profile(d_A, d_B, d_C, d_D, self._n_sys, self._n_row)

    def set_rho_device(self, d_A, d_B, d_C):
        if self._filt is not None:
            self._filt.set_rho_device(d_A, d_B, d_C)

    def set_eps_constant(self, eps_constant):
        if self._filt is not None:
            self._filt.set_eps_constant(eps_constant)

    def last_gpu_ms(self):
        return (self._filt or self._pasc).last_gpu_ms()

    def last_J(self):
        return self._filt.last_J() if self._filt is not None else -1
