"""2-D boundary-integral RCS solve path (GPU)."""
