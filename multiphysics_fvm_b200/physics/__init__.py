"""Physics modules (mirror of the reference's src/physics package)."""
