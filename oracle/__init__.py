"""Test infrastructure: the CPU oracle (checker only, never the product)."""
