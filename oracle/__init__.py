"""Oracle package marker (test infrastructure only)."""
