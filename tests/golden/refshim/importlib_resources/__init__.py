from importlib.resources import files  # noqa: F401
