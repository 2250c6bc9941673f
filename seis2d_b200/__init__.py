"""seis2d_b200: B200-native (sm_100a) forward modelling for SeisAcoMod2D.

The modelling path is the CUDA library ``libseis2d.so`` (built in-tree from
``seis2d_b200/csrc`` by ``seis2d_b200.build``) behind the C ABI of
``include/seis2d.h``.  This package is its Python host layer.
"""
from .api import Context, Model, Shot, Wave, derive_steps, modelling_module  # noqa: F401

__all__ = ["Context", "Model", "Shot", "Wave", "derive_steps", "modelling_module"]
