"""Test oracle for the swap search: CPU restatement and reference-engine harness (test infrastructure only)."""
