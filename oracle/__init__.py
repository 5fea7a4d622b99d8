"""CPU checkers for the ARGOT hot path (test infrastructure only; the
product package ``argot_b200`` never imports this)."""
