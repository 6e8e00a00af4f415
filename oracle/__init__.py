"""Test oracle and reference-build helpers (test infrastructure, not the product)."""
