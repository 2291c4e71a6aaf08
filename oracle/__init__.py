"""FP64 CPU oracle of the reference's propagate-and-retrieve path (test infrastructure only)."""
