"""Loader of the native library.  There is no fallback: the SAP step runs only
through libsapb.so, and loading fails loudly when it is missing."""

from __future__ import annotations

import ctypes
import threading

from . import _abi
from .build import LIB_PATH

_lock = threading.Lock()
_lib: ctypes.CDLL | None = None


class SapbError(RuntimeError):
    """A native entry point returned an error status."""

    def __init__(self, status: int, where: str, message: str = ""):
        self.status = int(status)
        super().__init__(f"{where} failed with status {status}: {message}")


def load() -> ctypes.CDLL:
    global _lib
    with _lock:
        if _lib is None:
            if not LIB_PATH.exists():
                raise RuntimeError(
                    f"{LIB_PATH} is missing: build it with `python -m sap_warp_b200.build` "
                    "(the SAP step has no non-native path)"
                )
            lib = ctypes.CDLL(str(LIB_PATH))
            _abi.bind(lib)
            if lib.sapb_abi_version() != _abi.SAPB_ABI_VERSION:
                raise RuntimeError("libsapb.so ABI version does not match the Python bindings")
            _lib = lib
        return _lib


def check(status: int, where: str) -> None:
    if status != _abi.SAPB_OK:
        msg = load().sapb_last_error()
        raise SapbError(status, where, msg.decode() if msg else "")
