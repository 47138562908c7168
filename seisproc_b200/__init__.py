"""seisproc_b200: B200-native Kirchhoff pre-stack time migration (PSTM).

A drop-in for SeisProc's PSTM hot path (processors/migration): the same call
signatures (``MigrationEngine.migrate_bin_full``, ``migrate_kirchhoff_full``,
``normalize_by_fold``, the ``BaseMigrator`` API) and ``kernel_backend``
selection, computed by hand-written sm_100a CUDA kernels in libseispstm.so.
"""
from .kernel_backend import (KernelBackend, get_backend_info, get_effective_backend,
                             get_global_backend, set_global_backend)
from .models import (MigrationConfig, MigrationGeometry, OutputGrid, SeismicData, VelocityModel,
                     VelocityType, WeightMode, InterpolationMode, TraveltimeMode,
                     create_3d_velocity, create_constant_velocity, create_from_rms_velocity)

__all__ = [
    "KernelBackend", "get_backend_info", "get_effective_backend", "get_global_backend",
    "set_global_backend", "MigrationConfig", "MigrationGeometry", "OutputGrid", "SeismicData",
    "VelocityModel", "VelocityType", "WeightMode", "InterpolationMode", "TraveltimeMode",
    "create_3d_velocity", "create_constant_velocity", "create_from_rms_velocity",
    "MigrationEngine", "migrate_kirchhoff_full", "normalize_by_fold", "PSTMPlan",
    "release_cached_memory",
]


def release_cached_memory(keep_bytes: int = 0) -> None:
    """Return the device memory that finished plans left in the library's pool
    (beyond ``keep_bytes``) on the current CUDA device to the driver."""
    from . import _lib
    _lib.check(_lib.lib().pstm_trim_memory(int(keep_bytes)))


def __getattr__(name):
    # torch-dependent operators are imported lazily so the models stay importable alone
    if name in ("migrate_kirchhoff_full", "normalize_by_fold", "PSTMPlan", "normalize_mute"):
        from . import kirchhoff
        return getattr(kirchhoff, name)
    if name == "MigrationEngine":
        from .engine import MigrationEngine
        return MigrationEngine
    raise AttributeError(name)
