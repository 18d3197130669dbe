"""Loading of the native libraries and the ctypes view of the C-ABI (include/nabladyn_b200.h).

``lib()`` returns ``libnabladyn_b200.so`` with its entry points typed; ``neighbor_ops()`` loads
the torch.library layer and returns ``torch.ops.nabladyn_neighbors``. Both raise
``RuntimeError`` when the libraries have not been built: there is no fallback path.
"""

from __future__ import annotations

import ctypes
from pathlib import Path
from threading import RLock

import torch

_LIB_DIR = Path(__file__).resolve().parent / "_lib"
CORE_PATH = _LIB_DIR / "libnabladyn_b200.so"
OPS_PATH = _LIB_DIR / "_nabladyn_neighbors_ops.so"

ND_OK, ND_EINVAL, ND_ECUDA = 0, 1, 2
ND_FLOAT32, ND_FLOAT64 = 0, 1
INVALID_CELL, NON_FINITE, OVERFLOW = 1, 2, 8

# Reentrant: neighbor_ops() loads the core library under the same lock.
_LOCK = RLock()
_lib: ctypes.CDLL | None = None
_ops_loaded = False

c_int32_p = ctypes.POINTER(ctypes.c_int32)
c_int64_p = ctypes.POINTER(ctypes.c_int64)
c_double_p = ctypes.POINTER(ctypes.c_double)


class NeighborBuffers(ctypes.Structure):
    _fields_ = [
        ("dims", ctypes.c_void_p),
        ("widths", ctypes.c_void_p),
        ("atom_bin", ctypes.c_void_p),
        ("bin_counts", ctypes.c_void_p),
        ("bin_offsets", ctypes.c_void_p),
        ("num_bin_slots", ctypes.c_int64),
        ("unordered_ids", ctypes.c_void_p),
        ("sorted_ids", ctypes.c_void_p),
        ("sorted_positions", ctypes.c_void_p),
        ("scan_temp", ctypes.c_void_p),
        ("scan_temp_bytes", ctypes.c_int64),
        ("pair_counts", ctypes.c_void_p),
        ("pair_offsets", ctypes.c_void_p),
        ("pair_total", ctypes.c_void_p),
        ("status", ctypes.c_void_p),
        ("pairs", ctypes.c_void_p),
        ("capacity", ctypes.c_int64),
        ("bits", ctypes.c_void_p),
        ("bits_numel", ctypes.c_int64),
    ]


class ReuseBuffers(ctypes.Structure):
    _fields_ = [
        ("reference_positions", ctypes.c_void_p),
        ("reference_cell", ctypes.c_void_p),
        ("limits", ctypes.c_void_p),
        ("reuse", ctypes.c_void_p),
        ("rebuild", ctypes.c_void_p),
        ("rebuild_count", ctypes.c_void_p),
    ]


class LJPairsArgs(ctypes.Structure):
    _fields_ = [
        ("dtype", ctypes.c_int),
        ("positions", ctypes.c_void_p),
        ("cell", ctypes.c_void_p),
        ("num_atoms", ctypes.c_int64),
        ("pairs", ctypes.c_void_p),
        ("capacity", ctypes.c_int64),
        ("atom_types", ctypes.c_void_p),
        ("num_types", ctypes.c_int32),
        ("sigma", ctypes.c_void_p),
        ("epsilon", ctypes.c_void_p),
        ("cutoff", ctypes.c_double),
        ("strain", ctypes.c_void_p),
        ("energy", ctypes.c_void_p),
        ("forces", ctypes.c_void_p),
        ("virial", ctypes.c_void_p),
        ("sigma_grad", ctypes.c_void_p),
        ("epsilon_grad", ctypes.c_void_p),
    ]


class LJBatchArgs(ctypes.Structure):
    _fields_ = [
        ("dtype", ctypes.c_int),
        ("frames", ctypes.c_int64),
        ("positions", ctypes.c_void_p),
        ("cells", ctypes.c_void_p),
        ("num_atoms", ctypes.c_int64),
        ("pairs", ctypes.c_void_p),
        ("capacity", ctypes.c_int64),
        ("atom_types", ctypes.c_void_p),
        ("num_types", ctypes.c_int32),
        ("sigma", ctypes.c_void_p),
        ("epsilon", ctypes.c_void_p),
        ("cutoff", ctypes.c_double),
        ("energy", ctypes.c_void_p),
        ("forces", ctypes.c_void_p),
        ("virial", ctypes.c_void_p),
        ("energy_grad", ctypes.c_void_p),
        ("forces_grad", ctypes.c_void_p),
        ("virial_grad", ctypes.c_void_p),
        ("sigma_grad", ctypes.c_void_p),
        ("epsilon_grad", ctypes.c_void_p),
    ]


class MDSystem(ctypes.Structure):
    _fields_ = [
        ("dtype", ctypes.c_int),
        ("num_atoms", ctypes.c_int64),
        ("num_types", ctypes.c_int32),
        ("small", ctypes.c_int32),
        ("dims", ctypes.c_int32 * 3),
        ("bricks_x", ctypes.c_int32),
        ("width", ctypes.c_int32),
        ("tile_capacity", ctypes.c_int32),
        ("cell", ctypes.c_double * 3),
        ("widths", ctypes.c_double * 3),
        ("cutoff", ctypes.c_double),
        ("radius", ctypes.c_double),
        ("timestep", ctypes.c_double),
        ("threshold_squared", ctypes.c_double),
        ("positions", ctypes.c_void_p),
        ("velocities", ctypes.c_void_p),
        ("forces", ctypes.c_void_p),
        ("inverse_masses", ctypes.c_void_p),
        ("masses", ctypes.c_void_p),
        ("images", ctypes.c_void_p),
        ("ids", ctypes.c_void_p),
        ("reference_positions", ctypes.c_void_p),
        ("shadow_positions", ctypes.c_void_p),
        ("shadow_velocities", ctypes.c_void_p),
        ("shadow_inverse_masses", ctypes.c_void_p),
        ("shadow_masses", ctypes.c_void_p),
        ("shadow_images", ctypes.c_void_p),
        ("shadow_ids", ctypes.c_void_p),
        ("cell_counts", ctypes.c_void_p),
        ("cell_offsets", ctypes.c_void_p),
        ("atom_cell", ctypes.c_void_p),
        ("slots", ctypes.c_void_p),
        ("unordered", ctypes.c_void_p),
        ("order", ctypes.c_void_p),
        ("scan_temp", ctypes.c_void_p),
        ("neighbors", ctypes.c_void_p),
        ("neighbor_counts", ctypes.c_void_p),
        ("pair_order", ctypes.c_void_p),
        ("rebuild", ctypes.c_void_p),
        ("rebuild_count", ctypes.c_void_p),
        ("status", ctypes.c_void_p),
        ("partials", ctypes.c_void_p),
        ("totals", ctypes.c_void_p),
        ("thermostat", ctypes.c_void_p),
        ("sigma", ctypes.c_void_p),
        ("epsilon", ctypes.c_void_p),
    ]


class Replica(ctypes.Structure):
    _fields_ = [
        ("atom_offset", ctypes.c_int64),
        ("list_offset", ctypes.c_int64),
        ("cell_offset", ctypes.c_int64),
        ("num_atoms", ctypes.c_int32),
        ("width", ctypes.c_int32),
        ("dims", ctypes.c_int32 * 3),
        ("steps_left", ctypes.c_int32),
        ("status", ctypes.c_int32),
        ("rebuild_count", ctypes.c_int32),
        ("cell", ctypes.c_float * 3),
        ("widths", ctypes.c_float * 3),
        ("cutoff", ctypes.c_float),
        ("radius", ctypes.c_float),
        ("threshold_squared", ctypes.c_float),
        ("timestep", ctypes.c_float),
        ("sigma", ctypes.c_float),
        ("epsilon", ctypes.c_float),
        ("energy", ctypes.c_double),
        ("thermostat", ctypes.c_double * 24),
    ]


class ReplicaPool(ctypes.Structure):
    _fields_ = [
        ("replicas", ctypes.c_void_p),
        ("positions", ctypes.c_void_p),
        ("velocities", ctypes.c_void_p),
        ("forces", ctypes.c_void_p),
        ("masses", ctypes.c_void_p),
        ("inverse_masses", ctypes.c_void_p),
        ("images", ctypes.c_void_p),
        ("reference_positions", ctypes.c_void_p),
        ("neighbors", ctypes.c_void_p),
        ("neighbor_counts", ctypes.c_void_p),
        ("sorted", ctypes.c_void_p),
        ("scratch", ctypes.c_void_p),
        ("cell_starts", ctypes.c_void_p),
        ("ordered_positions", ctypes.c_void_p),
    ]


class SchNetArgs(ctypes.Structure):
    _fields_ = [
        ("num_atoms", ctypes.c_int64),
        ("num_columns", ctypes.c_int64),
        ("interactions", ctypes.c_int32),
        ("num_types", ctypes.c_int32),
        ("gaussians", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
        ("cutoff", ctypes.c_double),
        ("positions", ctypes.c_void_p),
        ("cell", ctypes.c_void_p),
        ("pairs", ctypes.c_void_p),
        ("atom_types", ctypes.c_void_p),
        ("weights", ctypes.c_void_p),
        ("workspace", ctypes.c_void_p),
        ("energy", ctypes.c_void_p),
        ("forces", ctypes.c_void_p),
        ("virial", ctypes.c_void_p),
        ("status", ctypes.c_void_p),
    ]


class SchNetTangentArgs(ctypes.Structure):
    _fields_ = [
        ("num_atoms", ctypes.c_int64),
        ("num_columns", ctypes.c_int64),
        ("interactions", ctypes.c_int32),
        ("num_types", ctypes.c_int32),
        ("gaussians", ctypes.c_int32),
        ("block", ctypes.c_int32),
        ("cutoff", ctypes.c_double),
        ("weights", ctypes.c_void_p),
        ("workspace", ctypes.c_void_p),
        ("force_adjoint", ctypes.c_void_p),
        ("virial_adjoint", ctypes.c_void_p),
        ("v", ctypes.c_void_p),
        ("v_dot", ctypes.c_void_p),
        ("m", ctypes.c_void_p),
        ("m_dot", ctypes.c_void_p),
        ("m_bar", ctypes.c_void_p),
        ("m_dot_bar", ctypes.c_void_p),
        ("v_bar", ctypes.c_void_p),
        ("v_dot_bar", ctypes.c_void_p),
        ("pair_rows", ctypes.c_void_p),
        ("capacity", ctypes.c_int64),
        ("status", ctypes.c_void_p),
    ]


class SchNetAtomArgs(ctypes.Structure):
    _fields_ = [
        ("num_atoms", ctypes.c_int64),
        ("interactions", ctypes.c_int32),
        ("num_types", ctypes.c_int32),
        ("atom_types", ctypes.c_void_p),
        ("parameters", ctypes.c_void_p),
        ("gradient", ctypes.c_void_p),
        ("energy_adjoint", ctypes.c_void_p),
        ("workspace", ctypes.c_void_p),
    ]


class Integrator(ctypes.Structure):
    _fields_ = [
        ("dtype", ctypes.c_int),
        ("num_atoms", ctypes.c_int64),
        ("positions", ctypes.c_void_p),
        ("velocities", ctypes.c_void_p),
        ("forces", ctypes.c_void_p),
        ("masses", ctypes.c_void_p),
        ("images", ctypes.c_void_p),
        ("cell", ctypes.c_void_p),
        ("thermostat", ctypes.c_void_p),
        ("partials", ctypes.c_void_p),
        ("totals", ctypes.c_void_p),
        ("status", ctypes.c_void_p),
        ("timestep", ctypes.c_double),
        ("barostat", ctypes.c_void_p),
        ("virial", ctypes.c_void_p),
    ]


# name -> (argument types); every entry point returns int.
_SIGNATURES = {
    "nd_abi_version": [],
    "nd_neighbors_scan_temp_bytes": [ctypes.c_int64, c_int64_p],
    "nd_neighbors_count_first_frame": [
        ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_double,
        ctypes.POINTER(NeighborBuffers), ctypes.c_void_p,
    ],
    "nd_neighbors_fill_first_frame": [
        ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_double,
        ctypes.POINTER(NeighborBuffers), ctypes.c_void_p,
    ],
    "nd_neighbors_update": [
        ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_double,
        ctypes.c_double, ctypes.POINTER(ReuseBuffers), ctypes.POINTER(NeighborBuffers),
        ctypes.c_void_p,
    ],
    "nd_neighbors_build_no_alloc": [
        ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_double,
        ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p,
        ctypes.c_void_p, ctypes.c_void_p,
    ],
    "nd_lj_energy_force_virial": [ctypes.POINTER(LJPairsArgs), ctypes.c_void_p],
    "nd_lj_batch_forward": [ctypes.POINTER(LJBatchArgs), ctypes.c_void_p],
    "nd_lj_batch_parameter_backward": [ctypes.POINTER(LJBatchArgs), ctypes.c_void_p],
    "nd_md_import": [
        ctypes.POINTER(MDSystem), ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
        ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
    ],
    "nd_md_rebuild": [ctypes.POINTER(MDSystem), ctypes.c_void_p],
    "nd_md_forces": [ctypes.POINTER(MDSystem), ctypes.c_int, ctypes.c_void_p],
    "nd_md_step": [ctypes.POINTER(MDSystem), ctypes.c_int, ctypes.c_int, ctypes.c_void_p],
    "nd_md_run_small": [ctypes.POINTER(MDSystem), ctypes.c_int, ctypes.c_int, ctypes.c_void_p],
    "nd_md_step_phase": [
        ctypes.POINTER(MDSystem), ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
    ],
    "nd_md_step_launches": [ctypes.POINTER(MDSystem), c_int64_p],
    "nd_md_export": [
        ctypes.POINTER(MDSystem), ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
        ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
    ],
    "nd_md_kinetic": [ctypes.POINTER(MDSystem), ctypes.c_int, ctypes.c_void_p],
    "nd_md_partial_slots": [ctypes.POINTER(MDSystem), c_int64_p],
    "nd_md_graph_create": [ctypes.POINTER(MDSystem), ctypes.c_int, ctypes.c_int,
                           ctypes.POINTER(ctypes.c_void_p)],
    "nd_md_graph_launch": [ctypes.c_void_p, ctypes.c_void_p],
    "nd_md_graph_destroy": [ctypes.c_void_p],
    "nd_serve_run": [
        ctypes.POINTER(ReplicaPool), ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32,
        ctypes.c_int32, ctypes.c_void_p,
    ],
    "nd_schnet_energy_force_virial": [ctypes.POINTER(SchNetArgs), ctypes.c_void_p],
    "nd_schnet_tangent": [ctypes.POINTER(SchNetTangentArgs), ctypes.c_int32, ctypes.c_void_p],
    "nd_schnet_atoms": [ctypes.POINTER(SchNetAtomArgs), ctypes.c_int32, ctypes.c_int32,
                        ctypes.c_void_p],
    "nd_integrate_partial_slots": [ctypes.c_int64, c_int64_p],
    "nd_integrate_open": [ctypes.POINTER(Integrator), ctypes.c_int, ctypes.c_void_p],
    "nd_integrate_close": [ctypes.POINTER(Integrator), ctypes.c_int, ctypes.c_void_p],
    "nd_integrate_kinetic": [ctypes.POINTER(Integrator), ctypes.c_int, ctypes.c_void_p],
}

# name -> (argument types) of the entry points that return a byte count (int64, -1 on error).
_SIZES = {
    "nd_schnet_weight_bytes": [ctypes.c_int32, ctypes.c_int32],
    "nd_schnet_workspace_bytes": [ctypes.c_int64, ctypes.c_int64, ctypes.c_int32],
    "nd_schnet_atom_parameter_floats": [ctypes.c_int32, ctypes.c_int32],
    "nd_schnet_atom_workspace_bytes": [ctypes.c_int64, ctypes.c_int32],
    "nd_schnet_atom_offset": [ctypes.c_int64, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32],
}

# Every symbol include/nabladyn_b200.h declares.
EXPORTED = ("nd_last_error", *_SIGNATURES, *_SIZES)


def _missing(path: Path) -> RuntimeError:
    return RuntimeError(
        f"the nabladyn_b200 native library {path.name} is not built; run "
        "`python -m nabladyn_b200.csrc.build` (nvcc for sm_100a) first",
    )


def lib() -> ctypes.CDLL:
    """Return the C-ABI library, loaded once per process."""
    global _lib
    if _lib is None:
        with _LOCK:
            if _lib is None:
                if not CORE_PATH.exists():
                    raise _missing(CORE_PATH)
                loaded = ctypes.CDLL(str(CORE_PATH))
                loaded.nd_last_error.restype = ctypes.c_char_p
                loaded.nd_last_error.argtypes = []
                for name, argtypes in _SIGNATURES.items():
                    function = getattr(loaded, name)
                    function.restype = ctypes.c_int
                    function.argtypes = argtypes
                for name, argtypes in _SIZES.items():
                    function = getattr(loaded, name)
                    function.restype = ctypes.c_int64
                    function.argtypes = argtypes
                _lib = loaded
    return _lib


def neighbor_ops():
    """Return ``torch.ops.nabladyn_neighbors``, the reference's schemas over our kernels."""
    global _ops_loaded
    if not _ops_loaded:
        with _LOCK:
            if not _ops_loaded:
                lib()
                if not OPS_PATH.exists():
                    raise _missing(OPS_PATH)
                torch.ops.load_library(str(OPS_PATH))
                _ops_loaded = True
    return torch.ops.nabladyn_neighbors


class NativeError(RuntimeError):
    """A C-ABI call that returned an error code."""


def call(name: str, *args) -> None:
    """Call entry point ``name`` and raise ``NativeError`` with its message on failure."""
    native = lib()
    rc = getattr(native, name)(*args)
    if rc != ND_OK:
        message = native.nd_last_error().decode(errors="replace")
        raise NativeError(f"{name} failed ({rc}): {message}")


def stream_handle(device: torch.device) -> int:
    """The raw cudaStream_t of torch's current stream on ``device``."""
    return torch.cuda.current_stream(device).cuda_stream


def dtype_code(dtype: torch.dtype) -> int:
    if dtype == torch.float32:
        return ND_FLOAT32
    if dtype == torch.float64:
        return ND_FLOAT64
    raise TypeError("the native kernels take float32 or float64")


def ptr(tensor: torch.Tensor | None) -> int | None:
    """The device address of a contiguous tensor, or None."""
    if tensor is None:
        return None
    if not tensor.is_contiguous():
        raise ValueError("native kernels take contiguous tensors")
    return tensor.data_ptr()


__all__ = ("lib", "neighbor_ops", "call", "EXPORTED")
