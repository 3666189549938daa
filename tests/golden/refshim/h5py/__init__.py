"""Empty stand-in: HDF5 I/O is not on the template-matching path."""
