"""CPU oracle — test infrastructure only (see oracle/oracle.py); the product never imports this package."""
