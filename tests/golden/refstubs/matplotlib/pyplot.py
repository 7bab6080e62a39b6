"""Import stub for matplotlib.pyplot (annotations such as ``plt.Figure`` only)."""
from . import _Anything


def __getattr__(name):
    return _Anything()
