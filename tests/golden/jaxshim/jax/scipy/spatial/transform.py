"""jax.scipy.spatial.transform stand-in: SciPy's Rotation (same API, NumPy arrays)."""
from scipy.spatial.transform import Rotation  # noqa: F401
