"""despeckcl_b200: despeckCL's NL-SAR path, native to one NVIDIA B200 (sm_100a).

The public functions keep the names and signatures of despeckCL's Python
bindings; see ``api.py``.
"""
from .api import (  # noqa: F401
    DEFAULT_LOG_LEVELS,
    SELECT_MODES,
    DespeckclError,
    NlsarBatch,
    NlsarServer,
    Params,
    Stats,
    StatsCollection,
    boxcar,
    boxcar_device,
    goldstein,
    goldstein_device,
    lib,
    load_nlsar_stats_collection,
    nlsar,
    nlsar_insar,
    nlsar_insar_batch_device,
    nlsar_insar_device,
    nlinsar,
    nlinsar_device,
    nlsar_train,
    nlsar_train_insar,
    store_nlsar_stats_collection,
    stats_from_dissims,
    take_stage_timeouts,
)

__version__ = "0.1.0"
