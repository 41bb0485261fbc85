"""jax.scipy.linalg names the reference imports, from SciPy."""

from scipy.linalg import cho_solve, lu_factor, lu_solve, solve_triangular  # noqa: F401
