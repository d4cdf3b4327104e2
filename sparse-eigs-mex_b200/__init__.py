"""speigs on B200: thick-restart Lanczos ('sm' shift-invert, 'lm' direct)
behind the reference's C ABI.  The compute lives in lib/libspeigs.so (built
from csrc/); this package is the ctypes binding plus workload generators."""
from . import learned, shard, speigs, tune, workloads  # noqa: F401
from .speigs import LIB_PATH, Plan, load  # noqa: F401
