"""Stand-in for proxide.physics (TEST INFRASTRUCTURE ONLY)."""
