"""fastweavturb_b200 -- B200-native woven-turbulence field construction (drop-in for the
field-construction path of FastWeavTurb's `tube` program).

The product is the CUDA library ``libfwt.so`` behind the C-ABI in ``include/fwt.h``.  This
package is its thin ctypes binding (used by the tests, the benchmark and the learned
surrogate).  There is no CPU path: loading fails loudly when the library or a GPU is missing.
"""
from .api import (  # noqa: F401
    Context,
    FwtError,
    Params,
    fbb_signs,
    library,
    run_dir,
    sp_exponents,
    sp_separations,
)
from .configs import CONFIGS, Workload, build_workload  # noqa: F401
