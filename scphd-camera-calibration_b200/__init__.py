"""B200-native SC-PHD camera-calibration filter step.

The directory name is not a Python identifier; load it with `load_package()` from
the repository root helpers (bench.py, __graft_entry__.py, tests/conftest.py),
which registers it as the module `scphd_b200`.
"""
from .scphd import (COUNTER_NAMES, SCPHD_FP32, SCPHD_FP64, SCPHD_MIX_FITTED, SCPHD_MIX_MERGED,  # noqa: F401
                    JOB_DONE, JOB_QUEUED, JOB_RUNNING, SCPHDBatch, SCPHDCameraCalibration, SCPHDServer, ScphdConfig, ScphdError, ScphdFrame, kernel_launches,
                    config_from_file, device_bytes, load_library, merge_components, read_mat_frames,
                    write_mat_arrays, reference_defaults, systematic_resample)
from . import evaluate, scene  # noqa: F401
