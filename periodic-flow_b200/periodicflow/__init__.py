"""periodicflow -- B200 backend of the periodic pseudo-spectral Navier-Stokes solver.

Same public API as the reference package (``simulation.Solver``,
``space_solver``, ``time_integrator`` registry, ``math`` kernels), with the
right-hand side and the time loop running as sm_100a CUDA kernels behind the
C ABI of ``libpfb200.so``.  Selecting this package on ``PYTHONPATH`` is the
backend switch; ``PERIODICFLOW_BACKEND`` must be unset or ``cuda``.
"""
import logging
import os

try:
    from rich.console import Console
    from rich.logging import RichHandler
    _handler = RichHandler(console=Console(width=120), show_time=False, show_level=False,
                           show_path=False)
except ImportError:  # pragma: no cover - rich is optional here
    _handler = logging.StreamHandler()

logging.basicConfig(level=logging.INFO, format="%(asctime)s [%(levelname)s] %(message)s",
                    datefmt="%Y-%m-%d %H:%M:%S", handlers=[_handler])
logger = logging.getLogger("periodicflow")

BACKEND = os.environ.get("PERIODICFLOW_BACKEND", "cuda").lower()
if BACKEND != "cuda":
    raise ImportError(
        f"PERIODICFLOW_BACKEND={BACKEND!r}: this package is the CUDA backend; put the "
        "reference periodicflow package on PYTHONPATH for its CPU backend")
