"""Build-time WGSL-subset -> C++/CUDA translator for formula plugins."""

from .wgsl import TranslateError, TranslatedFormula, translate, translate_module  # noqa: F401
