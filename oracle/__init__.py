"""CPU oracle of the path-tracing hot path (test infrastructure only)."""
