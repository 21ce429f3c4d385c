from . import linalg, special, spatial  # noqa: F401
