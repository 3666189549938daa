"""Empty stand-in: MRC I/O is not on the template-matching path."""
