"""Dense boundary-operator assembly on the GPU, from Python.

The public names, arguments and ValueError texts follow bempp-rs's
``python/bempp/assembly/boundary.py`` (``BoundaryAssemblerOptions``,
``BoundaryAssembler.assemble`` returning a Fortran-ordered numpy matrix,
``assemble_singular`` returning SciPy CSR, ``create_laplace_assembler``), so code written
against the reference runs unchanged.  Beyond the reference:

* ``create_helmholtz_assembler`` wraps the C factory that the reference exports
  (src/bindings/boundary_assemblers.rs:168-210) but never wrapped in Python;
* ``set_precision`` picks FP64 or mixed FP32/FP64 regular quadrature;
* ``assemble_into_device`` fills a device buffer (a torch CUDA tensor, say) on a CUDA
  stream without a host round trip, and ``check_device`` reports whether such an
  assembly completed;
* phase timing, launch counts and host-copy statistics for measurement.
"""

from __future__ import annotations

import typing
import weakref
from enum import Enum

import numpy as np
import numpy.typing as npt
from scipy.sparse import csr_matrix

from bempp._lib import check as _check
from bempp._lib import ffi as _ffi
from bempp._lib import last_error as _last_error
from bempp._lib import lib as _lib
from bempp.function_space import FunctionSpace
from ndelement.reference_cell import ReferenceCellType

_rtypes = {
    np.float32: _lib.DType_F32,
    np.float64: _lib.DType_F64,
    np.complex64: _lib.DType_C32,
    np.complex128: _lib.DType_C64,
}
_dtypes = {j: i for i, j in _rtypes.items()}
_real = {np.float32: np.float32, np.float64: np.float64, np.complex64: np.float32,
         np.complex128: np.float64}


def _convert_to_scipy(rs_sparse_mat, dtype: typing.Type[np.floating]) -> csr_matrix:
    """Copy a library-owned CSR MatrixT into SciPy arrays, then release the MatrixT."""
    if rs_sparse_mat == _ffi.NULL:
        raise RuntimeError(_last_error())
    shape = (_lib.matrix_shape0(rs_sparse_mat), _lib.matrix_shape1(rs_sparse_mat))
    data = np.empty(_lib.matrix_csr_data_size(rs_sparse_mat), dtype=dtype)
    indices = np.empty(_lib.matrix_csr_indices_size(rs_sparse_mat), dtype=np.uintp)
    indptr = np.empty(_lib.matrix_csr_indptr_size(rs_sparse_mat), dtype=np.uintp)
    _lib.matrix_csr_data_copy(rs_sparse_mat, _ffi.cast("void*", data.ctypes.data))
    _lib.matrix_csr_indices_copy(rs_sparse_mat, _ffi.cast("uintptr_t*", indices.ctypes.data))
    _lib.matrix_csr_indptr_copy(rs_sparse_mat, _ffi.cast("uintptr_t*", indptr.ctypes.data))
    _lib.matrix_t_free(rs_sparse_mat)
    return csr_matrix((data, indices, indptr), shape=shape)


class OperatorType(Enum):
    """Which boundary operator to assemble (values of the C enum OperatorType)."""

    SingleLayer = _lib.OperatorType_SingleLayer
    DoubleLayer = _lib.OperatorType_DoubleLayer
    AdjointDoubleLayer = _lib.OperatorType_AdjointDoubleLayer
    Hypersingular = _lib.OperatorType_Hypersingular
    ElectricField = _lib.OperatorType_ElectricField
    MagneticField = _lib.OperatorType_MagneticField


class Precision(Enum):
    """Arithmetic of the regular far-pair quadrature (addition)."""

    FP64 = _lib.Precision_FP64
    Mixed = _lib.Precision_Mixed


# Dense outputs of at least this many bytes are allocated page-locked (set to None to
# always allocate pageable numpy memory).
PINNED_OUTPUT_MIN_BYTES = 16 << 20


class _PageLockedBlock:
    """Owner of one page-locked block of the library's cache, exposed to numpy through
    ``__array_interface__`` (column-major); the block returns to the cache when the last
    array viewing it is gone."""

    def __init__(self, shape, dtype):
        self._dtype = np.dtype(dtype)
        self._shape = tuple(int(x) for x in shape)
        nbytes = int(np.prod(self._shape)) * self._dtype.itemsize
        self._ptr = _lib.bempp_host_alloc(nbytes)
        if self._ptr == _ffi.NULL:
            raise MemoryError(_last_error())
        item = self._dtype.itemsize
        self.__array_interface__ = {
            "shape": self._shape, "typestr": self._dtype.str,
            "data": (int(_ffi.cast("uintptr_t", self._ptr)), False),
            "strides": (item, item * self._shape[0]), "version": 3}

    def __del__(self):
        ptr = getattr(self, "_ptr", None)
        if ptr is not None and ptr != _ffi.NULL:
            try:
                _lib.bempp_host_free(ptr)
            except Exception:  # interpreter shutdown
                pass


def _host_output(shape, dtype):
    """Column-major output array for ``assemble``.

    Large matrices live in page-locked blocks of the library's cache: the library then
    writes the finished columns into them by DMA while later columns are still being
    computed, with no staging copy, and a block freed by one result is reused by the
    next.  Every entry is overwritten by the assembly.
    """
    nbytes = int(np.prod(shape)) * np.dtype(dtype).itemsize
    if PINNED_OUTPUT_MIN_BYTES is not None and nbytes >= PINNED_OUTPUT_MIN_BYTES:
        try:
            return np.asarray(_PageLockedBlock(shape, dtype))
        except MemoryError:  # page-locking refused: pageable memory
            pass
    return np.zeros(shape, dtype=dtype, order="F")


class BoundaryAssemblerOptions(object):
    """Quadrature and precision settings of an assembler.

    Once an assembler has been created from an options object, the object is frozen:
    the setters raise ValueError."""

    def __init__(self):
        self._read_only = False
        self._rs_options = _lib.boundary_assembler_options_new()
        # freed when the object goes, or at interpreter exit while the library is still
        # loaded
        weakref.finalize(self, _lib.boundary_assembler_options_t_free, self._rs_options)

    def set_regular_quadrature_degree(self, cell: ReferenceCellType, degree: int):
        """Number of points of the rule used on well-separated cell pairs of this cell
        type (the reference calls it the degree)."""
        if self._read_only:
            raise ValueError("Cannot edit options already being used by an assembler")
        if not _lib.boundary_assembler_options_has_regular_quadrature_degree(
            self._rs_options, cell.value
        ):
            raise ValueError(f"Invalid cell type: {cell}")
        _lib.boundary_assembler_options_set_regular_quadrature_degree(
            self._rs_options, cell.value, degree
        )

    def regular_quadrature_degree(self, cell: ReferenceCellType) -> int:
        """Points of the regular rule on this cell type."""
        if not _lib.boundary_assembler_options_has_regular_quadrature_degree(
            self._rs_options, cell.value
        ):
            raise ValueError(f"Invalid cell type: {cell}")
        return _lib.boundary_assembler_options_get_regular_quadrature_degree(
            self._rs_options, cell.value
        )

    def set_singular_quadrature_degree(
        self, cell0: ReferenceCellType, cell1: ReferenceCellType, degree: int
    ):
        """1-D Gauss order of the Duffy rules used on cell pairs that share a vertex."""
        if self._read_only:
            raise ValueError("Cannot edit options already being used by an assembler")
        if not _lib.boundary_assembler_options_has_singular_quadrature_degree(
            self._rs_options, cell0.value, cell1.value
        ):
            raise ValueError(f"Invalid cell pair: {cell0} and {cell1}")
        _lib.boundary_assembler_options_set_singular_quadrature_degree(
            self._rs_options, cell0.value, cell1.value, degree
        )

    def singular_quadrature_degree(self, cell0: ReferenceCellType, cell1: ReferenceCellType) -> int:
        """1-D Gauss order of the Duffy rules of this pair of cell types."""
        if not _lib.boundary_assembler_options_has_singular_quadrature_degree(
            self._rs_options, cell0.value, cell1.value
        ):
            raise ValueError(f"Invalid cell pair: {cell0} and {cell1}")
        return _lib.boundary_assembler_options_get_singular_quadrature_degree(
            self._rs_options, cell0.value, cell1.value
        )

    def set_batch_size(self, batch_size: int):
        """Cell-block size option (kept for API compatibility; the GPU kernels tile
        cells in blocks of 32 whatever it is)."""
        if self._read_only:
            raise ValueError("Cannot edit options already being used by an assembler")
        _lib.boundary_assembler_options_set_batch_size(self._rs_options, batch_size)

    def batch_size(self) -> int:
        """The cell-block size option."""
        return _lib.boundary_assembler_options_get_batch_size(self._rs_options)

    def set_precision(self, precision: Precision):
        """Set the arithmetic of the regular far-pair quadrature (addition)."""
        if self._read_only:
            raise ValueError("Cannot edit options already being used by an assembler")
        _lib.boundary_assembler_options_set_precision(self._rs_options, precision.value)

    def precision(self) -> Precision:
        """Arithmetic of the regular far-pair quadrature."""
        return Precision(_lib.boundary_assembler_options_get_precision(self._rs_options))


class BoundaryAssembler(object):
    """Assembles one operator (kernel, operator type, scalar type) for pairs of spaces."""

    def __init__(self, options: BoundaryAssemblerOptions, rs_assembler, owned: bool = True):
        """Wrap a BoundaryAssemblerT; freezes ``options``."""
        if rs_assembler == _ffi.NULL:
            raise ValueError(_last_error())
        self.options = options
        self.options._read_only = True
        self._rs_assembler = rs_assembler
        if owned:
            weakref.finalize(self, _lib.boundary_assembler_t_free, rs_assembler)

    def _check_spaces(self, trial_space: FunctionSpace, test_space: FunctionSpace):
        ok = (trial_space.dtype, test_space.dtype)
        allowed = (self.dtype, _real[self.dtype])
        assert ok[0] in allowed and ok[1] in allowed, "space and assembler dtypes differ"

    def assemble(
        self, trial_space: FunctionSpace, test_space: FunctionSpace
    ) -> npt.NDArray[np.floating]:
        """The dense test x trial matrix as a Fortran-ordered numpy array (page-locked
        when large, so that finished columns arrive by DMA while the rest is computed)."""
        self._check_spaces(trial_space, test_space)
        output = _host_output((test_space.global_size, trial_space.global_size), self.dtype)
        _check(
            _lib.boundary_assembler_assemble_into_memory_ex(
                self._rs_assembler,
                trial_space._rs_space,
                test_space._rs_space,
                _ffi.cast("void*", output.ctypes.data),
            ),
            "assemble",
        )
        return output

    def assemble_into_device(self, trial_space: FunctionSpace, test_space: FunctionSpace,
                             out, stream=None, check: bool = False):
        """Fill a device buffer with the dense matrix (addition).

        ``out`` is anything with ``data_ptr()`` (a torch CUDA tensor) or a raw device
        address, with room for test.global_size x trial.global_size elements of the
        assembler's dtype stored column by column: a torch tensor of shape
        (n_trial, n_test) is the natural fit.  ``stream`` is a cudaStream_t as an int
        (``torch.cuda.current_stream().cuda_stream``); None means the legacy default
        stream.  The call returns as soon as the work is enqueued; with ``check=True``
        it waits for the stream and raises if the assembly did not complete
        (``check_device``).
        """
        self._check_spaces(trial_space, test_space)
        ptr = out.data_ptr() if hasattr(out, "data_ptr") else int(out)
        _check(
            _lib.boundary_assembler_assemble_into_device(
                self._rs_assembler, trial_space._rs_space, test_space._rs_space,
                _ffi.cast("void*", ptr), _ffi.cast("void*", int(stream or 0))),
            "assemble_into_device",
        )
        if check:
            check_device(stream)

    def assemble_singular(
        self, trial_space: FunctionSpace, test_space: FunctionSpace
    ) -> csr_matrix:
        """Only the entries of cell pairs that share a vertex (the Duffy-rule part), as
        SciPy CSR; an empty matrix when every such entry is negligible."""
        self._check_spaces(trial_space, test_space)
        return _convert_to_scipy(
            _lib.boundary_assembler_assemble_singular(
                self._rs_assembler,
                trial_space._rs_space,
                test_space._rs_space,
            ),
            self.dtype,
        )

    def set_timing(self, enabled: bool = True):
        """Record CUDA events around the geometry, regular and singular phases."""
        _lib.boundary_assembler_set_timing(self._rs_assembler, enabled)

    def phase_times(self) -> typing.List[float]:
        """Milliseconds of the phases of the last timed assembly."""
        buf = np.zeros(8, dtype=np.float64)
        n = _lib.boundary_assembler_phase_times(
            self._rs_assembler, _ffi.cast("double*", buf.ctypes.data), 8)
        return [float(x) for x in buf[:n]]

    def host_copy_stats(self) -> typing.Dict[str, float]:
        """Host side of the last host-memory assembly: DMA wait and host copy times (ms),
        copy groups, assembly chunks, copy threads, page prefault time, and for page-locked
        destinations the device time to the end of the kernels and of the last DMA."""
        buf = np.zeros(8, dtype=np.float64)
        n = _lib.boundary_assembler_host_copy_stats(
            self._rs_assembler, _ffi.cast("double*", buf.ctypes.data), 8)
        keys = ("dma_wait_ms", "host_copy_ms", "groups", "chunks", "threads", "prefault_ms",
                "compute_ms", "dma_end_ms")
        return {k: float(v) for k, v in zip(keys[:n], buf[:n])}

    def launch_count(self) -> int:
        """Kernel launches enqueued by the last assembly."""
        return _lib.boundary_assembler_last_launch_count(self._rs_assembler)

    @property
    def dtype(self):
        """Scalar type of the matrices this assembler produces."""
        return _dtypes[_lib.boundary_assembler_dtype(self._rs_assembler)]


def create_laplace_assembler(
    operator_type: OperatorType,
    options: typing.Optional[BoundaryAssemblerOptions] = None,
    dtype: typing.Type[np.floating] = np.float64,
):
    """Assembler of a Laplace operator (f32 or f64), G(x, y) = 1 / (4 pi |x - y|)."""
    options = BoundaryAssemblerOptions() if options is None else options
    return BoundaryAssembler(
        options,
        _lib.laplace_boundary_assembler_new(
            options._rs_options, operator_type.value, _rtypes[dtype]
        ),
    )


def create_helmholtz_assembler(
    operator_type: OperatorType,
    wavenumber: float,
    options: typing.Optional[BoundaryAssemblerOptions] = None,
    dtype: typing.Type[np.complexfloating] = np.complex128,
):
    """Assembler of a Helmholtz operator (c64 or c128) with wavenumber ``wavenumber``,
    G(x, y) = exp(i k |x - y|) / (4 pi |x - y|)."""
    options = BoundaryAssemblerOptions() if options is None else options
    real = np.float32 if dtype == np.complex64 else np.float64
    k = np.array([wavenumber], dtype=real)
    ctype = "float*" if real == np.float32 else "double*"
    return BoundaryAssembler(
        options,
        _lib.helmholtz_boundary_assembler_new(
            _ffi.cast(ctype, k.ctypes.data), options._rs_options, operator_type.value,
            _rtypes[dtype]
        ),
    )


def check_device(stream=None):
    """Wait for ``stream`` and raise RuntimeError if a device-memory assembly launched
    since the last check did not complete: a block of the regular kernels gave up waiting
    for its shared-memory tile copies (a bounded wait) and wrote none of its entries."""
    _check(_lib.bempp_device_status(_ffi.cast("void*", int(stream or 0))), "device assembly")
