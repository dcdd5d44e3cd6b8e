"""Python host side of the B200 SIMPLE solver: case builders and the C-ABI binding."""
from . import cases  # noqa: F401
from .abi import (  # noqa: F401
    AxisimError, Solver, build, lib, multiblock, resolve_bc, PREC_FP64, PREC_MIXED, EXPORTS,
)
