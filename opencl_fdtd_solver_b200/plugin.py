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
    """Anything callable as ``cb(engine)``; the engine calls it once per step.

    Registered as a source, it is called between the two half steps: H is already
    at n+1/2 and ``engine.t`` reads the half-step time.  Registered as a monitor,
    it is called once the step is complete, with E at n+1 and ``t`` advanced.
    """

    def __call__(self, fdtd: Any) -> None: ...


class SourceMonitorMixin:
    """``add_source`` / ``add_monitor`` and their ``clear_*`` counterparts.

    An engine using this mixin owns two lists, ``_sources`` and ``_monitors``,
    created in its constructor; the methods only append to or empty them.
    """

    _sources: list
    _monitors: list

    def add_source(self, source: StepCallback) -> StepCallback:
        """Append ``source``, called with the engine between the H and E half steps."""
        if not callable(source):
            raise TypeError(f"source must be callable, got {type(source)!r}")
        self._sources.append(source)
        return source

    def add_monitor(self, monitor: StepCallback) -> StepCallback:
        """Append ``monitor``, called with the engine at the end of each step."""
        if not callable(monitor):
            raise TypeError(f"monitor must be callable, got {type(monitor)!r}")
        self._monitors.append(monitor)
        return monitor

    def clear_sources(self) -> None:
        """Forget every source added so far."""
        self._sources.clear()

    def clear_monitors(self) -> None:
        """Forget every monitor added so far."""
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
