"""TEST INFRASTRUCTURE — the CPU oracle (see oracle/oracle.py). Never imported
by the product package."""
