"""CPU oracle package: test infrastructure only (the checker, never the product)."""
