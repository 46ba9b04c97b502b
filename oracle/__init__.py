"""Oracle package (test infrastructure only)."""
