"""Import stub for matplotlib, used only when importing the reference package
to generate golden fixtures. Plotting is never exercised."""


class _Anything:
    def __getattr__(self, name):
        return _Anything()

    def __call__(self, *a, **k):
        return _Anything()


def __getattr__(name):
    return _Anything()
