"""Test-side checkers for the B200 CKKS engine (never imported by the product)."""
