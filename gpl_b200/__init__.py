"""gpl_b200: a B200-native engine for vyges-gpl's `global_placement` command."""
from .design import Design  # noqa: F401
