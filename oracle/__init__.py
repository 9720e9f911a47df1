"""TEST INFRASTRUCTURE: the oracle package (checkers only, never the product)."""
