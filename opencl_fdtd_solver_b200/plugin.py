"""Source/monitor registration and the backend registry.

``StepCallback`` and ``SourceMonitorMixin`` keep the reference contract
(``opencl_fdtd_solver/plugin.py:13-53``): a source callback ``cb(fdtd)`` runs after
the H update with ``fdtd.t`` at the half step, a monitor callback runs after the
full step with fields and ``t`` advanced, and non-callables raise ``TypeError``.

The reference has no backend registry; ``BACKENDS`` / ``get_backend`` add one so
that code selecting an engine by name (``"cuda"``) finds ``CUDAFDTD``.
"""

from __future__ import annotations

from typing import Any, Callable, Protocol, runtime_checkable


@runtime_checkable
class StepCallback(Protocol):
    """Callable invoked once per timestep with the solver instance.

    Sources run after the H update and before the E update.
    Monitors run after the full Yee step (fields and ``t`` advanced).
    """

    def __call__(self, fdtd: Any) -> None: ...


class SourceMonitorMixin:
    """Registration API for per-step sources and monitors.

    Concrete solvers initialise ``_sources`` and ``_monitors`` in ``__init__``.
    """

    _sources: list
    _monitors: list

    def add_source(self, source: StepCallback) -> StepCallback:
        """Register ``source(fdtd)``; it runs after every H update."""
        if not callable(source):
            raise TypeError(f"source must be callable, got {type(source)!r}")
        self._sources.append(source)
        return source

    def add_monitor(self, monitor: StepCallback) -> StepCallback:
        """Register ``monitor(fdtd)``; it runs after every full step."""
        if not callable(monitor):
            raise TypeError(f"monitor must be callable, got {type(monitor)!r}")
        self._monitors.append(monitor)
        return monitor

    def clear_sources(self) -> None:
        """Remove all registered source callbacks."""
        self._sources.clear()

    def clear_monitors(self) -> None:
        """Remove all registered monitor callbacks."""
        self._monitors.clear()


BACKENDS: dict[str, Callable[..., Any]] = {}


def register_backend(name: str, cls: Callable[..., Any]) -> Callable[..., Any]:
    """Register an engine class under ``name`` (later registrations replace earlier)."""
    BACKENDS[str(name).lower()] = cls
    return cls


def get_backend(name: str = "cuda") -> Callable[..., Any]:
    """Return the engine class registered under ``name``."""
    try:
        return BACKENDS[str(name).lower()]
    except KeyError:
        raise KeyError(f"unknown FDTD backend {name!r}; registered: {sorted(BACKENDS)}") from None
