"""Import stub for scikit-image, used only when importing the reference package
to generate golden fixtures. Phantom-image objects are never built."""
from matplotlib import _Anything  # noqa: F401  (stub package beside this one)

data = _Anything()
transform = _Anything()
