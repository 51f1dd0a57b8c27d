"""Public entry point for the locked stable profile."""

from ..profiles import StableSBLPlan, make_stable_plan

__all__ = ["StableSBLPlan", "make_stable_plan"]
