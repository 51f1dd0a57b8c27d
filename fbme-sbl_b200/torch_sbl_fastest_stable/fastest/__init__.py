"""Public entry point for the locked minimum-latency profile."""

from ..profiles import FastestSBLPlan, make_fastest_plan

__all__ = ["FastestSBLPlan", "make_fastest_plan"]
