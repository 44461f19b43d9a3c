"""structure_b200: a B200-native (sm_100a) engine for STRUCTURE's per-sweep
MCMC hot path, behind the C ABI of include/stgpu.h (libstgpu.so)."""
from .api import (Context, Data, Chain, Batch, Model, StError, model_defaults, lib,  # noqa: F401
                  LAYOUT_AUTO, LAYOUT_U8, LAYOUT_B2G)

__all__ = ["Context", "Data", "Chain", "Batch", "Model", "StError", "model_defaults", "lib"]
