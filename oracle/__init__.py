"""Oracle of the model-evaluation path (test infrastructure only)."""
