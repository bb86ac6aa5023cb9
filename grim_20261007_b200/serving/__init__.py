"""Continuous-batching request engine for RCS solves (HBM-budget admission, factor cache)."""
from .engine import FactorCache, Request, ServingEngine, synthetic_stream  # noqa: F401
