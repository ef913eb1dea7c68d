"""`native_core` of the reference (native_core/__init__.py), on the GPU: the
`formation_core` module with the same names and call signatures."""
from . import formation_core  # noqa: F401
