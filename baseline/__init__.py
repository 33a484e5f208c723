"""Baselines measured beside the engine (not part of the product)."""
