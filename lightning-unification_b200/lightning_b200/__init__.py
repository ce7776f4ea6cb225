"""lightning_b200 — B200-native state-vector engine behind the lightning.qubit surface.

* ``lightning_b200.lightning_qubit_ops`` — pybind11 module with the reference's
  classes (StateVectorC64/C128, MeasurementsC64/C128, observables.*,
  algorithms.*), backed by libb200sv.
* ``lightning_b200.capi`` — ctypes view of the C ABI (include/b200sv.h).
* ``lightning_b200.batch`` / ``lightning_b200.autograd`` — the batched engine and
  its torch.autograd.Function.

Importing a native piece that was not built raises ImportError: there is no CPU
fallback anywhere in this package.
"""
from pathlib import Path

__version__ = "0.1.0"
PACKAGE_DIR = Path(__file__).resolve().parent


def build(verbose: bool = False, force: bool = False) -> None:
    """Compile libb200sv.so (nvcc, sm_100a) and the pybind11 module in place."""
    from . import _build
    _build.build_all(verbose=verbose, force=force)
