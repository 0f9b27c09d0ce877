"""Backends of the GRG matmul path.  Only ``b200`` exists; import it explicitly (it needs torch)."""
