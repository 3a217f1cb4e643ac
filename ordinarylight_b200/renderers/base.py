"""Renderer implementation identity and protocol.

When the reference package ``ordinarylight`` has already been imported, its
own ``RendererImplementation``/``RendererImplementationInfo``/
``RendererProtocol`` (ordinarylight/renderers/base.py:16-70) are reused so
``isinstance`` checks in reference code see this package's renderers as
reference implementations.  Otherwise structurally identical definitions
are provided here.  ``graphics_api="cuda"`` extends the reference's
``GraphicsApi`` literal (a static type hint only; nothing checks it at run
time).
"""

from __future__ import annotations

from dataclasses import dataclass
import sys
from typing import Any, ClassVar, Mapping, Protocol, runtime_checkable

_reference = sys.modules.get("ordinarylight.renderers.base")

if _reference is not None:
    RendererImplementation = _reference.RendererImplementation
    RendererImplementationInfo = _reference.RendererImplementationInfo
    RendererProtocol = _reference.RendererProtocol
else:
    @dataclass(frozen=True)
    class RendererImplementationInfo:
        """Stable identity of a concrete renderer implementation."""

        name: str
        family: str
        graphics_api: str

    class RendererImplementation:
        """Nominal base for renderers with discoverable identity."""

        implementation: ClassVar[RendererImplementationInfo]

        @classmethod
        def implementation_info(cls) -> RendererImplementationInfo:
            return cls.implementation

    @runtime_checkable
    class RendererProtocol(Protocol):
        """Structural renderer contract: linear-HDR ``render_frame`` plus ``close``."""

        available_outputs: tuple
        config: Any
        device: Any
        last_timings: Mapping

        def render_frame(self, scene, camera, width: int, height: int, *, samples: int | None = None,
                         frame_index: int = 0):
            ...

        def close(self) -> None:
            ...

__all__ = ["RendererImplementation", "RendererImplementationInfo", "RendererProtocol"]
