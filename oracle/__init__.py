"""Test infrastructure: the CPU oracle (C restatement + patched reference harness)."""
