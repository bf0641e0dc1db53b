"""NL-SAR oracle: test infrastructure only (see pyoracle.py)."""
