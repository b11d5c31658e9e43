"""Analysis wrappers over the RMSD plans."""
