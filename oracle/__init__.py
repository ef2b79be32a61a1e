"""Test-only oracles for SORT's ray-query path. Never imported by the product."""
