"""Kernel backend selection for the PSTM path.

Mirrors the reference's selection interface (processors/kernel_backend.py:31-133:
``KernelBackend`` enum, a process-global preference with
``set_global_backend``/``get_global_backend``, and ``get_effective_backend``).
The reference enum values ``auto``/``python``/``metal_cpp`` are accepted;
``cuda_sm100`` is added.  ``AUTO`` and ``CUDA_SM100`` select the sm_100a
kernels.  There is deliberately no CPU or Metal path: ``PYTHON`` and
``METAL_CPP`` raise ``ValueError`` instead of silently falling back, and the
CUDA backend raises ``RuntimeError`` when no CUDA device or library is present.
"""
from __future__ import annotations

import logging
from enum import Enum
from typing import Any, Dict, Optional, Union

logger = logging.getLogger(__name__)


class KernelBackend(Enum):
    AUTO = "auto"
    PYTHON = "python"
    METAL_CPP = "metal_cpp"
    CUDA_SM100 = "cuda_sm100"


_global_backend: KernelBackend = KernelBackend.AUTO


def _coerce(b: Union[KernelBackend, str, None]) -> Optional[KernelBackend]:
    if b is None or isinstance(b, KernelBackend):
        return b
    if hasattr(b, "value"):  # a reference KernelBackend member
        b = b.value
    try:
        return KernelBackend(str(b).lower())
    except ValueError as e:
        raise ValueError(f"Unknown kernel backend: {b!r}") from e


def set_global_backend(backend: Union[KernelBackend, str]) -> None:
    global _global_backend
    _global_backend = _coerce(backend)
    logger.info("Global kernel backend set to: %s", _global_backend.value)


def get_global_backend() -> KernelBackend:
    return _global_backend


def is_cuda_available() -> bool:
    try:
        import torch
        return bool(torch.cuda.is_available())
    except Exception:  # pragma: no cover - torch import failure
        return False


def get_effective_backend(requested: Union[KernelBackend, str, None] = None) -> KernelBackend:
    """Resolve the backend for a PSTM call; always the CUDA sm_100a kernels."""
    b = _coerce(requested) or _global_backend
    if b in (KernelBackend.PYTHON, KernelBackend.METAL_CPP):
        raise ValueError(
            f"kernel_backend={b.value!r} is not provided by seisproc_b200: the PSTM path runs "
            "only on the CUDA sm_100a kernels (use 'auto' or 'cuda_sm100')")
    return KernelBackend.CUDA_SM100


def require_cuda(requested: Union[KernelBackend, str, None] = None) -> KernelBackend:
    b = get_effective_backend(requested)
    if not is_cuda_available():
        raise RuntimeError("seisproc_b200 PSTM requires a CUDA device (sm_100a); none is available")
    return b


def get_backend_info() -> Dict[str, Any]:
    return {
        "global_backend": _global_backend.value,
        "effective_backend": KernelBackend.CUDA_SM100.value,
        "python_available": False,
        "metal_cpp_available": False,
        "cuda_sm100_available": is_cuda_available(),
    }
