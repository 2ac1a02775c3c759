"""B200-native device path of rcsr: batched bytecode scoring, fused-adjoint
batched LM/IRLS constant fitting, input gradients and the implicit metric,
behind the reference's `rc_*` C ABI (include/rcsr_b200.h).

The directory name is not a Python identifier; import it with
`importlib.import_module("the-rule-and-compass_b200")`.
"""
from . import expr, host  # noqa: F401
from .device import GpuEvaluator, GenomePool, DeviceError, MultiEvaluator  # noqa: F401
from .device import lib as cuda_lib  # noqa: F401
from .host import compile_program, gpu_fit_plan, Population, pack_plans  # noqa: F401
from .host import DEFAULT_VARIATION_OPS, width_for, FitLedger  # noqa: F401
from .host import refit_finalists_exact, soa_eval, soa_sse  # noqa: F401
from .search import GenerationLoop  # noqa: F401
