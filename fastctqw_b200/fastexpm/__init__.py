"""Drop-in for FastCTQW.fastexpm (FastCTQW/fastexpm/__init__.py:1)."""
from ._wrapper import ExpMatComplex64, ExpMatComplex128, ExpMatFloat32, ExpMatFloat64

__all__ = ["ExpMatFloat32", "ExpMatFloat64", "ExpMatComplex64", "ExpMatComplex128"]
