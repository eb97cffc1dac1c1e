"""CPU oracle for the flip dynamics (TEST INFRASTRUCTURE ONLY; see pyoracle.py)."""
