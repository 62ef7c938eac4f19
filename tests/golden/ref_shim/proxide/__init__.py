"""Stand-in for the proxide package (TEST INFRASTRUCTURE ONLY)."""
