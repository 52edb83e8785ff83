"""Scheme selectors: named callables that a setup dict puts in ``space_schemes``.

In this package the space schemes are evaluated inside the fused CUDA stage
kernel, not as separate array functions; each selector carries the enum that
the kernel dispatch uses (``_fvm_id``) and refuses direct host calls.
"""


def selector(kind: str, name: str, enum, doc: str):
    def f(*_args, **_kwargs):
        raise TypeError(f"{name} selects a scheme of the fused CUDA stage kernel; it is evaluated on the "
                        "device by Simulation / solver.run, not called on host arrays")
    f.__name__ = f.__qualname__ = name
    f.__doc__ = doc
    f._fvm_id = (kind, enum)
    return f
