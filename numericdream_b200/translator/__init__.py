"""Build-time WGSL-subset -> C++/CUDA translator for formula plugins."""

from .wgsl import TranslateError, TranslatedFormula, translate  # noqa: F401
