"""B200-native electron-repulsion-integral engine with a gbasis-compatible host API."""
from .contractions import GeneralizedContractionShell, is_shell  # noqa: F401

__all__ = ["GeneralizedContractionShell", "is_shell"]
