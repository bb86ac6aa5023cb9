"""Body-of-revolution RCS solve path (GPU)."""
