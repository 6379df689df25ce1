"""ctypes mirror of include/statecraft_b200.h and the loader of the native library.

The native library is built in-tree (``statecraft_b200/_native/libstatecraft_b200.so``)
by ``statecraft_b200.build``.  There is no Python fallback: when the library is
missing every engine entry point raises ``NativeLibraryMissing``.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

SC_ABI_VERSION = 2

SC_OK = 0
SC_EINVAL = -1
SC_EUNSUPPORTED = -2
SC_ESTATE = -3
SC_ENOMEM = -4
SC_ECUDA = -5
SC_ETIMEOUT = -6

SC_C128 = 0
SC_C64 = 1

SC_OP_SINGLE = 1
SC_OP_CNOT = 2
SC_OP_TWO = 3
SC_OP_DIAG2 = 4
SC_OP_SWAP = 5
SC_OP_MULTI = 6
SC_OP_MEASURE = 7
SC_OP_RX = 16
SC_OP_RY = 17
SC_OP_RZ = 18
SC_OP_RZZ = 19

SC_MAX_KRAUS = 8
SC_DEFAULT_MAX_QUBITS = 32


class ScOp(ctypes.Structure):
    _fields_ = [
        ("kind", ctypes.c_int32),
        ("q0", ctypes.c_int32),
        ("q1", ctypes.c_int32),
        ("param", ctypes.c_int32),
        ("mask", ctypes.c_uint64),
        ("m", ctypes.c_double * 32),
    ]


class ScChannel(ctypes.Structure):
    _fields_ = [
        ("after_op", ctypes.c_int64),
        ("target", ctypes.c_int32),
        ("n_kraus", ctypes.c_int32),
        ("kraus", (ctypes.c_double * 8) * SC_MAX_KRAUS),
    ]


class ScConfig(ctypes.Structure):
    _fields_ = [
        ("dtype", ctypes.c_int32),
        ("fusion", ctypes.c_int32),
        ("tile_qubits", ctypes.c_int32),
        ("sweep_budget", ctypes.c_int32),
        ("max_qubits", ctypes.c_int32),
        ("timing", ctypes.c_int32),
        ("device_mem_limit", ctypes.c_int64),
        ("autotune", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
    ]


assert ctypes.sizeof(ScOp) == 280
assert ctypes.sizeof(ScConfig) == 40
assert ctypes.sizeof(ScChannel) == 16 + 8 * 8 * SC_MAX_KRAUS


class NativeLibraryMissing(RuntimeError):
    """The CUDA extension is not built or cannot be loaded; there is no CPU fallback."""


_P = ctypes.POINTER
_c_void_pp = _P(ctypes.c_void_p)

# name -> (restype, argtypes); every symbol declared in include/statecraft_b200.h
SIGNATURES = {
    "sc_version": (ctypes.c_int32, []),
    "sc_last_error": (ctypes.c_char_p, []),
    "sc_create": (ctypes.c_int32, [ctypes.c_int32, _P(ScConfig), _c_void_pp]),
    "sc_destroy": (ctypes.c_int32, [ctypes.c_void_p]),
    "sc_set_noise": (ctypes.c_int32, [ctypes.c_void_p, _P(ScChannel), ctypes.c_int64,
                                      ctypes.c_uint64, ctypes.c_int32]),
    "sc_run": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_int32, _P(ScOp), ctypes.c_int64,
                                _P(ctypes.c_double), ctypes.c_uint64, ctypes.c_int32]),
    "sc_get_state": (ctypes.c_int32, [ctypes.c_void_p, _P(ctypes.c_double), ctypes.c_int64]),
    "sc_default_measured_qubits": (ctypes.c_int32, [ctypes.c_void_p, _P(ctypes.c_int32),
                                                    ctypes.c_int32]),
    "sc_sample": (ctypes.c_int32, [ctypes.c_void_p, _P(ctypes.c_int32), ctypes.c_int32,
                                   ctypes.c_int64, ctypes.c_uint64, ctypes.c_int32,
                                   _P(ctypes.c_double), _P(ctypes.c_int32)]),
    "sc_probabilities": (ctypes.c_int32, [ctypes.c_void_p, _P(ctypes.c_int32), ctypes.c_int32,
                                          _P(ctypes.c_double)]),
    "sc_expect_pauli": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_int32, _P(ctypes.c_uint64),
                                         _P(ctypes.c_uint64), _P(ctypes.c_double),
                                         _P(ctypes.c_double)]),
    "sc_adjoint_forward": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_int32, _P(ScOp),
                                            ctypes.c_int64, _P(ctypes.c_double), ctypes.c_int64,
                                            ctypes.c_int32, _P(ctypes.c_uint64),
                                            _P(ctypes.c_uint64), _P(ctypes.c_double),
                                            _P(ctypes.c_double)]),
    "sc_adjoint_backward": (ctypes.c_int32, [ctypes.c_void_p, _P(ctypes.c_double),
                                             ctypes.c_int64]),
    "sc_qaoa_batch_create": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64,
                                              _P(ctypes.c_int32), ctypes.c_int32,
                                              _P(ctypes.c_double), _P(ctypes.c_double),
                                              ctypes.c_int32, _P(ctypes.c_void_p)]),
    "sc_qaoa_batch_set_angles": (ctypes.c_int32, [ctypes.c_void_p, _P(ctypes.c_double),
                                                  _P(ctypes.c_double)]),
    "sc_qaoa_batch_run": (ctypes.c_int32, [ctypes.c_void_p]),
    "sc_qaoa_batch_energies": (ctypes.c_int32, [ctypes.c_void_p, _P(ctypes.c_double),
                                                _P(ctypes.c_double)]),
    "sc_qaoa_batch_info": (ctypes.c_int32, [ctypes.c_void_p, _P(ctypes.c_int32),
                                            _P(ctypes.c_int32), _P(ctypes.c_double),
                                            _P(ctypes.c_double)]),
    "sc_qaoa_batch_destroy": (ctypes.c_int32, [ctypes.c_void_p]),
    "sc_trajectories": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_int32, _P(ScOp),
                                         ctypes.c_int64, _P(ScChannel), ctypes.c_int64,
                                         ctypes.c_int64, ctypes.c_uint64, ctypes.c_int64,
                                         ctypes.c_uint64, _P(ctypes.c_int32),
                                         _P(ctypes.c_int32), _P(ctypes.c_double)]),
    "sc_trajectories_info": (ctypes.c_int32, [ctypes.c_void_p, _P(ctypes.c_int32),
                                              _P(ctypes.c_int32), _P(ctypes.c_int32),
                                              _P(ctypes.c_double)]),
    "sc_kernel_stats": (ctypes.c_int32, [ctypes.c_void_p, _P(ctypes.c_int64),
                                         _P(ctypes.c_double), _P(ctypes.c_double),
                                         ctypes.c_int32]),
    "sc_kernel_class_name": (ctypes.c_char_p, [ctypes.c_int32]),
    "sc_reset_kernel_stats": (ctypes.c_int32, [ctypes.c_void_p]),
    "sc_stream": (ctypes.c_void_p, [ctypes.c_void_p]),
    "sc_sample_static": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32,
                                          ctypes.c_int64, ctypes.c_uint64, ctypes.c_void_p,
                                          ctypes.c_void_p, ctypes.c_void_p]),
    "sc_last_plan_stats": (ctypes.c_int32, [ctypes.c_void_p, _P(ctypes.c_int64),
                                            _P(ctypes.c_int64), _P(ctypes.c_int64)]),
    "sc_debug_entry_folds": (ctypes.c_int32, [ctypes.c_int32, _P(ScOp), ctypes.c_int64,
                                              ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                              ctypes.c_double, _P(ctypes.c_int64)]),
    "sc_debug_plan_order": (ctypes.c_int32, [ctypes.c_int32, _P(ScOp), ctypes.c_int64,
                                             ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                             ctypes.c_double, _P(ctypes.c_int64),
                                             _P(ctypes.c_int64), _P(ctypes.c_int64),
                                             _P(ctypes.c_int64), _P(ctypes.c_int64)]),
    "sc_debug_emulate_sweeps": (ctypes.c_int32, [ctypes.c_int32, _P(ScOp), ctypes.c_int64,
                                                 ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                                 ctypes.c_double, _P(ctypes.c_double)]),
    "sc_debug_check_exchanges": (ctypes.c_int32, [ctypes.c_int32, _P(ScOp), ctypes.c_int64,
                                                  ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                                  ctypes.c_int32, _P(ctypes.c_int64)]),
    "sc_debug_check_tile_tensors": (ctypes.c_int32, [ctypes.c_int32, _P(ScOp), ctypes.c_int64,
                                                     ctypes.c_int32, ctypes.c_int32,
                                                     ctypes.c_int32, ctypes.c_int32,
                                                     ctypes.c_int64, _P(ctypes.c_int64)]),
    "sc_debug_emulate_slots": (ctypes.c_int32, [ctypes.c_int32, _P(ScOp), ctypes.c_int64,
                                                ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                                ctypes.c_double, _P(ctypes.c_int64),
                                                _P(ctypes.c_int32), ctypes.c_int64,
                                                _P(ctypes.c_uint8), _P(ctypes.c_double)]),
}

PACKAGE_DIR = Path(__file__).resolve().parent
LIB_PATH = PACKAGE_DIR / "_native" / "libstatecraft_b200.so"

_lib = None


def library_path() -> Path:
    override = os.environ.get("STATECRAFT_B200_LIB")
    return Path(override) if override else LIB_PATH


def load() -> ctypes.CDLL:
    """Loads the native library once and binds every declared symbol."""
    global _lib
    if _lib is not None:
        return _lib
    path = library_path()
    if not path.exists():
        raise NativeLibraryMissing(
            f"native library not found at {path}; run `python -m statecraft_b200.build`")
    try:
        lib = ctypes.CDLL(str(path))
    except OSError as exc:
        raise NativeLibraryMissing(f"cannot load {path}: {exc}") from exc
    for name, (restype, argtypes) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = restype
        fn.argtypes = argtypes
    if lib.sc_version() != SC_ABI_VERSION:
        raise NativeLibraryMissing(
            f"ABI version mismatch: library {lib.sc_version()} != {SC_ABI_VERSION}")
    _lib = lib
    return lib


class IllegalArgumentException(ValueError):
    """java.lang.IllegalArgumentException counterpart (SC_EINVAL)."""


class UnsupportedOperationException(NotImplementedError):
    """java.lang.UnsupportedOperationException counterpart (SC_EUNSUPPORTED)."""


class IllegalStateException(RuntimeError):
    """java.lang.IllegalStateException counterpart (SC_ESTATE)."""


class EngineError(RuntimeError):
    """Device-side failure (SC_ENOMEM, SC_ECUDA, SC_ETIMEOUT)."""

    def __init__(self, msg: str, status: int):
        super().__init__(msg)
        self.status = status


def raise_for(rc: int, lib: ctypes.CDLL | None = None) -> None:
    """Maps a status to the exception type the Java engine throws."""
    if rc >= 0:
        return
    lib = lib or load()
    raw = lib.sc_last_error()
    msg = raw.decode() if raw else f"status {rc}"
    if rc == SC_EINVAL:
        raise IllegalArgumentException(msg)
    if rc == SC_EUNSUPPORTED:
        raise UnsupportedOperationException(msg)
    if rc == SC_ESTATE:
        raise IllegalStateException(msg)
    raise EngineError(msg, rc)
