"""Golden cases for the grouped aggregate: the reference's seeded tests
regenerated (reference_cases.py, jrandom.py) and their expected outputs
(expected.json, written by make_golden.py)."""
