"""Exception types of the engine.

``CapabilityError`` is the reference's own class when ``qarp`` is importable (so engine
code that catches ``qarp.errors.CapabilityError`` sees the engine's rejections), else a
local class with the same base: a ``ValueError`` subclass (reference:
src/qarp/errors.py:9).
"""
try:  # pragma: no cover - exercised only where the reference package is installed
    from qarp.errors import CapabilityError  # type: ignore
except Exception:  # noqa: BLE001
    class CapabilityError(ValueError):
        """A declared capability is incompatible with the engine, circuit, or call."""

        command = None


class CudaError(RuntimeError):
    """A CUDA runtime failure inside the engine library."""


__all__ = ["CapabilityError", "CudaError"]
