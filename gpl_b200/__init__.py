"""gpl_b200: a B200-native engine for vyges-gpl's `global_placement` command.

The command runs through the C ABI in libgpl_b200.so (include/gpl.h): the placer's
construction on the host, the initial placement's solve and the Nesterov loop on the device.
"""
from .design import Design  # noqa: F401


def global_placement(design, args, router=None, device=0, poisson="mixed"):
    """The reference's `run::global_placement` (src/run.rs:115) on one B200."""
    from .engine import global_placement as _gp
    return _gp(design, args, router, device, poisson)
