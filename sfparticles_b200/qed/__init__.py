"""QED event generation method, chosen as in the reference (qed/__init__.py:1-6):
``SFPARTICLES_OPTICAL_DEPTH=1`` selects the optical-depth method, otherwise
rejection sampling.  ``set_method`` switches it for species created afterwards."""
from os import getenv

_use_optical_depth = getenv("SFPARTICLES_OPTICAL_DEPTH") == "1"


def use_optical_depth() -> bool:
    return _use_optical_depth


def set_method(method: str) -> None:
    """'rs' (rejection sampling) or 'od' (optical depth)."""
    global _use_optical_depth
    if method not in ("rs", "od"):
        raise ValueError("method must be 'rs' or 'od'")
    _use_optical_depth = method == "od"
