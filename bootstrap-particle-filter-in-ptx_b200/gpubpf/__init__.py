"""gpubpf — B200-native (sm_100a) bootstrap particle filter for the SV model.

Python face of libgpubpf.so (C ABI in include/gpu_bpf.h). The package
directory is not importable by its hyphenated parent name; put
``<repo>/bootstrap-particle-filter-in-ptx_b200`` on ``sys.path`` and
``import gpubpf``.
"""
from ._lib import BpfError, BpfResult, BpfTickRecord, LIB_PATH, load  # noqa: F401
from .filter import GpuBpf, debug_normals, debug_pcg32, run_rmse  # noqa: F401
from .batch import GpuBpfBatch  # noqa: F401
from .grad import BpfBatchLoglik, BpfLoglik, GradTape, ancestors_from_children, bpf_batch_loglik, bpf_loglik  # noqa: F401
from .imm import Imm, build_grid  # noqa: F401
from .apf import GpuApf, apf_run_rmse  # noqa: F401
from .smc2 import Smc2  # noqa: F401
from . import configs, dgp  # noqa: F401

TILE = 4096
