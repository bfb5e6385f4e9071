"""Timed CPU baseline: the reference's own solve, run end to end.

TEST / BASELINE INFRASTRUCTURE ONLY (used by bench.py's CPU-baseline leg and
its ``--impl reference`` arm).  ``oracle/Makefile`` compiles the reference's
pybind11 kernels from the reference sources and stages the reference
package beside them in ``oracle/_ref/momwire``; this module imports that
package and times its public call, ``BSplineSolver(**kw).
compute_port_solution()`` (``bspline.py:4053``): the chunked dense fill
(``_compute_Z_operator``, ``bspline.py:3702``, the C++ kernels with
OpenMP) and LAPACK ``zgesv`` through scipy (``_solve_with_kcl_ports``,
``bspline.py:2971``).  Nothing here is the product's code, and the product
package is not imported.

The thread counts must be set before numpy is first imported (OpenBLAS
reads them once): ``pin_threads()`` does that and returns the count.
"""

from __future__ import annotations

import glob
import os
import sys
import time
from pathlib import Path

HERE = Path(__file__).resolve().parent
REF_DIR = HERE / "_ref"


def pin_threads(n: int | None = None) -> int:
    """Use every host core for OpenMP and OpenBLAS (call before numpy is
    imported)."""
    if n is None:
        try:
            n = len(os.sched_getaffinity(0))
        except AttributeError:
            n = os.cpu_count() or 1
    for var in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS"):
        os.environ[var] = str(n)
    return n


def load_reference_kernels():
    """Import the reference's compiled ``_accelerators`` from oracle/_ref."""
    so = glob.glob(str(REF_DIR / "_accelerators*.so"))
    if not so:
        raise ImportError("reference kernels not built: run `make -C oracle REF=...`")
    sys.path.insert(0, str(REF_DIR))
    try:
        import _accelerators  # noqa: E402
    finally:
        sys.path.pop(0)
    return _accelerators


def import_reference():
    """The reference package staged by ``oracle/Makefile`` (its own Python
    modules with its compiled kernels); raises if it is missing or its
    kernels do not load."""
    if not (REF_DIR / "momwire" / "__init__.py").exists():
        raise ImportError("reference package not staged: run `make -C oracle REF=...`")
    if str(REF_DIR) not in sys.path:
        sys.path.insert(0, str(REF_DIR))
    import momwire  # noqa: E402

    if not Path(momwire.__file__).resolve().is_relative_to(REF_DIR.resolve()):
        raise ImportError(f"a different momwire is importable first: {momwire.__file__}")
    if not momwire.accelerated:
        raise ImportError("the reference's C++ kernels did not load")
    return momwire


def time_solve(momwire, kw):
    """One cold ``compute_port_solution()`` of a fresh reference solver.
    Returns (PortSolution, {"total_s", "fill_s", "solve_s"}); the fill and
    LU+solve phases are timed by wrapping the instance's own
    ``_compute_Z_operator`` and ``_solve_with_kcl_ports``."""
    s = momwire.BSplineSolver(**kw)
    phases = {"fill_s": 0.0, "solve_s": 0.0}

    def timed(name, fn):
        def run(*a, **k):
            t0 = time.perf_counter()
            try:
                return fn(*a, **k)
            finally:
                phases[name] += time.perf_counter() - t0

        return run

    s._compute_Z_operator = timed("fill_s", s._compute_Z_operator)
    s._solve_with_kcl_ports = timed("solve_s", s._solve_with_kcl_ports)
    t0 = time.perf_counter()
    sol = s.compute_port_solution()
    phases["total_s"] = time.perf_counter() - t0
    return sol, phases


def loaded_native_objects():
    """Shared objects mapped into this process (from /proc/self/maps)."""
    out = set()
    try:
        with open("/proc/self/maps") as f:
            for line in f:
                path = line.split()[-1] if len(line.split()) >= 6 else ""
                if path.endswith(".so") or ".so." in path:
                    out.add(path)
    except OSError:
        pass
    return sorted(out)
